#!/usr/bin/env python
"""Benchmark of the apg-sgm B200 engine (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload NAME]

A step is one stereo pair through the whole dense-matching pipeline (aux, cost + right-image
WTA, SGM sweeps + WTA, confidence / LR / fill / median).  `value` is W*H*D per second over all
ranks with the pair already resident in HBM and the L2 flushed between steps; `e2e` is the same
metric through the public session API (apg_session_process) with host buffers, the
host->device and device->host copies inside every step.  Multi-GPU runs are independent
replicas (the pipeline has no exchange step): every rank processes its own pairs, the device
time is the max over ranks.  `--impl reference` times the reference's own CPU implementation
(oracle/_ref, its AVX2/OpenMP Packed backend) on the host cores instead.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    # name: (mode, PairSpec args, label, configuration overrides)
    "fast720": (0, (1280, 720, 128, 12, 0, 120, 0.0), "fast_1280x720_d128", {}),
    "balanced640": (1, (640, 480, 64, 8, 4, 60, 0.0), "balanced_640x480_d64", {}),
    "balanced720": (1, (1280, 720, 128, 12, 0, 120, 0.0), "balanced_1280x720_d128", {}),
    "hq1080": (2, (1920, 1080, 256, 16, 0, 240, 0.2), "highquality_1920x1080_d256", {}),
    "hq720": (2, (1280, 720, 128, 12, 0, 120, 0.2), "highquality_1280x720_d128", {}),
    "balanced1080": (1, (1920, 1080, 256, 16, 0, 240, 0.0), "balanced_1920x1080_d256", {}),
    "fast1080": (0, (1920, 1080, 256, 16, 0, 240, 0.0), "fast_1920x1080_d256", {}),
    "kitti1242": (1, (1242, 375, 192, 12, 0, 180, 0.0), "balanced_1242x375_d192", {}),
    # hierarchical coarse-to-fine search range (HierarchicalConfig defaults: R = 4, NearestValid)
    "balanced720_hier": (1, (1280, 720, 128, 12, 0, 120, 0.0), "balanced_1280x720_d128_hierarchical",
                         {"hier_enable": 1}),
    "hq1080_hier": (2, (1920, 1080, 256, 16, 0, 240, 0.2), "highquality_1920x1080_d256_hierarchical",
                    {"hier_enable": 1}),
}
MODE_NAMES = {0: "Fast", 1: "Balanced", 2: "HighQuality"}


_SP_NAMES = {"legacy": 0, "curv_gate": 1, "conf_gate": 2, "stabilized": 3}
_IP_NAMES = {"legacy": 0, "shadow_reclass": 1}


def _scope_of(args):
    """(sp_method, sp_param, ip_method, ip_gap) from --subpixel NAME[:PARAM] and --inpaint NAME[:GAP]."""
    sp, _, spp = args.subpixel.partition(":")
    ip, _, ipg = args.inpaint.partition(":")
    return _SP_NAMES[sp], float(spp or 0.0), _IP_NAMES[ip], int(ipg or 32)


def _scope_label(args) -> dict:
    return {} if _scope_of(args) == (0, 0.0, 0, 32) else {"subpixel": args.subpixel, "inpaint": args.inpaint}


def metric_name(mode: int, w: int, h: int, D: int, over=None) -> str:
    kind = f"{MODE_NAMES[mode]}, hierarchical" if (over or {}).get("hier_enable") else MODE_NAMES[mode]
    return f"W*H*D/s at {w}x{h} D={D} ({kind}, bit-exact)"


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _profile_traffic(kernel: str, workload: str):
    """dram read+write bytes per launch from the committed ncu summary, if one exists."""
    f = ROOT / "profiles" / f"{kernel.replace('+', '_')}_{workload}.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


_SAMPLER_CHILD = r"""
import sys, time
path, bus, idx = sys.argv[1], sys.argv[2], int(sys.argv[3])
import pynvml as nv
nv.nvmlInit()
try:
    h = nv.nvmlDeviceGetHandleByPciBusId(bus) if bus else nv.nvmlDeviceGetHandleByIndex(idx)
except Exception:
    h = nv.nvmlDeviceGetHandleByIndex(idx)
smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
with open(path, "w", buffering=1) as f:
    while True:
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
        f.write(f"{time.monotonic()} {sm} {smax} {rs}\n")
        time.sleep(0.002)
"""


class ClockSampler:
    """SM clock and clock-event reasons of this rank's GPU, read through NVML every ~2 ms by a
    separate process that writes timestamped samples to a file (reads only; no setting is
    touched).  Nothing runs in the benchmark's own process meanwhile, so the timed launches never
    wait for a sampling thread.  mark() records monotonic-clock marks around the timed region so
    its samples can be told apart from the rest of the sampled window (the per-launch profile and
    the end-to-end legs that follow it, all with the GPU busy)."""

    REASON_BITS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
                   "sw_power_cap": 0x4}

    def __init__(self, device_index: int):
        self.dev = device_index
        self.marks = {}
        self.proc = None
        self.path = None

    def start(self):
        import tempfile
        bus = ""
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.dev)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
        except Exception:
            pass
        fd, self.path = tempfile.mkstemp(prefix="apg_clocks_", suffix=".txt")
        os.close(fd)
        try:
            self.proc = subprocess.Popen([sys.executable, "-c", _SAMPLER_CHILD, self.path, bus, str(self.dev)],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def _samples(self):
        out = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = line.split()
                    if len(parts) == 4:
                        try:
                            out.append((float(parts[0]), float(parts[1]), float(parts[2]), int(parts[3])))
                        except ValueError:
                            pass
        except OSError:
            pass
        return out

    def wait_first(self, timeout: float = 15.0):
        """Block until the first sample has been written, so the timed region is covered."""
        t0 = time.time()
        while self.proc and self.proc.poll() is None and time.time() - t0 < timeout:
            if os.path.getsize(self.path) > 0:
                return
            time.sleep(0.005)

    def mark(self, name: str):
        self.marks[name] = time.monotonic()

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        samples = self._samples()
        try:
            os.unlink(self.path)
        except OSError:
            pass
        if not samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml sampler unavailable"], "samples": 0}
        t0, t1 = self.marks.get("timed_start"), self.marks.get("timed_end")
        timed = [x for x in samples if t0 is not None and t1 is not None and t0 <= x[0] <= t1]
        busy = [x for x in samples if t0 is not None and x[0] >= t0]
        use = timed or busy
        reasons = sorted({n for x in use for n, bit in self.REASON_BITS.items() if x[3] & bit})
        return {"sm_mhz": statistics.median(x[1] for x in use) if use else None,
                "sm_max_mhz": max(x[2] for x in use) if use else None,
                "reasons": reasons, "samples": len(use), "samples_in_timed_region": len(timed),
                "window": "timed region" if timed else "timed region through the end-to-end legs",
                "source": "nvml (separate process)"}


def _volume_bytes(cfg, tuning) -> float:
    """Bytes per voxel of the volume the sweeps read, as the engine lays it out: one at 256 padded
    disparities for the census-only Fast volume and for the aggregated volume of one aggregation
    pass (tuning cost8: 0 = at 256, 1 = never, 2 = also at 128; 32 lanes per chain), else two."""
    t = dict(tuning)
    Dp = (cfg.max_disparity - cfg.min_disparity + 63) // 64 * 64
    fast_census = (not cfg.agg_enable and cfg.census_type == 1 and not cfg.use_ad and not cfg.use_grad
                   and not cfg.prior_enable and not cfg.hier_enable and not t.get("fast_fused", 0)
                   and t.get("cost_kernel", 0) != 1)
    one_pass = bool(cfg.agg_enable) and cfg.agg_iterations <= 1
    if t.get("cost8", 0) == 1 or t.get("sgm_lanes", 0) not in (0, 32) or not (fast_census or one_pass):
        return 2.0
    return 1.0 if Dp == 256 or (Dp == 128 and t.get("cost8", 0) == 2) else 2.0


def _algorithmic_bytes(name: str, w: int, h: int, D: int, volume_source: bool, npath: int = 4,
                       vb: float = 2.0) -> float:
    """Bytes a launch of `name` must move by design: the stage-boundary traffic of the kernel with
    u16 path sums and vb bytes per voxel of the volume the sweeps read (see _volume_bytes); a
    volume-fed sweep reads that volume once."""
    n = w * h
    vol = n * D * vb if volume_source else 0.0
    nfirst = npath - 1
    nin = 3  # Path8: five first-phase buffers folded into one before the last sweep
    return {
        "sgm_first": nfirst * (n * D * 2.0 + vol),    # every first-phase sweep writes its own sums
        "sgm_fold5": n * D * 12.0,                    # Path8: read 5 buffers, write 1
        "sgm_last_wta": nin * n * D * 2.0 + vol + n * 12,  # read the partial sums, write the WTA maps
        "cost+crossH": n * D * 2.0,                   # write the horizontally aggregated volume
        "crossV": n * D * (2.0 + vb),                 # read T, write C
        "cost": n * D * vb,                           # write the raw volume
    }.get(name, 0.0)


def run_reference(args, wl):
    """The reference CPU path (oracle/_ref) on the host cores, rank 0 only."""
    from oracle import oracle as O
    from apg_sgm_b200 import synthetic as S
    mode, spec, label, over = wl
    spec = S.PairSpec(*spec)
    L, R, _ = S.make_pair(spec, S.SEED_BASE)
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libapg_ref.so not built"}))
        return
    cfg = O.config(mode, spec.max_disparity, volume_backend=2, **over)  # Packed: the AVX2/OpenMP path
    O.set_experimental(*_scope_of(args), reference=True)  # the reference's scopes on this thread
    sess = O.RefSession(cfg, bounded_reuse=True)
    for _ in range(args.warmup):
        sess.process(L, R)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r = sess.process(L, R)
        times.append(time.perf_counter() - t0)
        assert r["status"] == 0
    vox = spec.width * spec.height * spec.max_disparity
    total = sum(times)
    value = vox * args.steps / total
    cores = O.ref_threads()
    print(json.dumps({
        "impl": "reference", "metric": metric_name(mode, spec.width, spec.height, spec.max_disparity, over),
        "value": value, "unit": "voxels/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": {"workload": label, "mode": MODE_NAMES[mode], "width": spec.width, "height": spec.height,
                   "max_disparity": spec.max_disparity, "backend": "Packed (AVX2/OpenMP)", **_scope_label(args)},
        "cpu_baseline": {"value": value, "unit": "voxels/s", "cores": cores, "kind": "reference",
                         "sample": f"{args.steps} pairs {spec.width}x{spec.height} D{spec.max_disparity} "
                                   f"{MODE_NAMES[mode]}, reference StereoSession Packed backend"},
        "e2e": {"value": value, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


SERVED_SIZES = [(640, 480, 64, 8, 4, 60), (1242, 375, 192, 12, 0, 180), (1280, 720, 128, 12, 0, 120),
                (1920, 1080, 256, 16, 0, 240)]


def _pinned(a):
    """A page-locked copy of a numpy array (host memory the copy engines read and write directly);
    the returned array keeps its pinned storage alive."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


def _served_stream(n, rate, seed):
    """n requests: (arrival s, size index, mode, pool slot); Poisson arrivals at `rate` pairs/s
    (rate 0: all at t = 0); sizes uniform over the four shapes; modes 70/20/10 Balanced/Fast/HQ."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, n) if rate > 0 else np.zeros(n)
    t = np.cumsum(gaps) - (gaps[0] if rate > 0 else 0.0)
    size = rng.integers(0, len(SERVED_SIZES), n)
    mode = rng.choice([1, 0, 2], size=n, p=[0.7, 0.2, 0.1])
    slot = rng.integers(0, 2, n)
    return list(zip(t.tolist(), size.tolist(), mode.tolist(), slot.tolist()))


def _out_pool(n_per_size=64):
    """Caller-owned page-locked result buffers, reused round-robin per size (a server's clients
    hand it their own output memory; fresh pageable arrays would add first-touch page faults and
    a staging copy to every request).  At most `slots` requests write at a time, all close in queue order, so a ring of 64
    per size never has two writers on one buffer."""
    pool = {}
    for si, (w, h, *_) in enumerate(SERVED_SIZES):
        pool[si] = [{"disparity": _pinned(np.zeros((h, w), np.float32)),
                     "confidence": _pinned(np.zeros((h, w), np.float32)),
                     "invalid_reason": _pinned(np.zeros((h, w), np.uint8)),
                     "reliable_mask": _pinned(np.zeros((h, w), np.uint8))}
                    for _ in range(n_per_size)]
    return pool


_OUT = {}


def _serve_stream(srv, pool, stream):
    """Submits every request at its arrival time (a submitter thread) and collects latencies."""
    import threading as th
    if not _OUT:
        _OUT.update(_out_pool())
    st0 = srv.stats()
    tickets = [None] * len(stream)
    lat = [0.0] * len(stream)
    t0 = time.perf_counter()

    def submitter():
        for i, (ta, si, mode, sl) in enumerate(stream):
            d = t0 + ta - time.perf_counter()
            if d > 0:
                time.sleep(d)
            L, R = pool[(si, mode, sl)]
            ring = _OUT[si]
            tickets[i] = srv.submit(L, R, mode=mode, max_disparity=SERVED_SIZES[si][2], out=ring[i % len(ring)])

    th_sub = th.Thread(target=submitter)
    th_sub.start()
    for i in range(len(stream)):
        while tickets[i] is None:
            time.sleep(0.0005)
        _, lat[i] = srv.wait(tickets[i])
    t_end = time.perf_counter()
    th_sub.join()
    st = srv.stats()
    lat = np.array(lat)
    span = t_end - t0
    return {"pairs_per_s": len(stream) / span, "p50_ms": float(np.percentile(lat, 50)),
            "p95_ms": float(np.percentile(lat, 95)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "span_s": span, "peak_in_flight": st["peak_in_flight"],
            "evictions": st["evictions"] - st0["evictions"], "peak_reserved_gb": st["peak_reserved_bytes"] / 2 ** 30}


def _bucket_device_ms(apg, pool, reps=5):
    """Device time of one pair alone for every (size, mode) of the stream: inputs resident in HBM,
    CUDA events on the engine's stream around each run, median of `reps`."""
    import torch
    dev = torch.device("cuda", 0)
    out = {}
    for si, (w, h, D, *_) in enumerate(SERVED_SIZES):
        o = [torch.empty((h, w), dtype=dt, device=dev) for dt in (torch.float32, torch.float32, torch.uint8, torch.uint8)]
        for mode in (0, 1, 2):
            L, R = (torch.from_numpy(a).to(dev) for a in pool[(si, mode, 0)])
            e = apg.Engine(apg.config_from_mode(mode, D))
            es = torch.cuda.ExternalStream(e.stream, device=dev)
            torch.cuda.synchronize()
            times = []
            for k in range(reps + 2):
                t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                t0.record(es)
                e.process_device(L.data_ptr(), R.data_ptr(), w, h, w, 1, *(t.data_ptr() for t in o))
                t1.record(es)
                e.sync()
                if k >= 2:
                    times.append(t0.elapsed_time(t1))
            out[(si, mode)] = float(np.median(times))
            e.close()
    return out


def _warm_server(apg, slots, pool):
    """A server whose pools hold `slots` warm engines for every (mode, size) of the stream."""
    srv = apg.Server(slots=slots, hbm_budget_gb=120.0)
    for si, (w, h, D, *_) in enumerate(SERVED_SIZES):
        for mode in (0, 1, 2):
            srv.reserve(w, h, mode=mode, max_disparity=D, count=slots)
    warm = _served_stream(4 * slots * len(SERVED_SIZES), 0, 1)
    _serve_stream(srv, pool, warm)
    return srv


def _served_pool():
    from apg_sgm_b200 import synthetic as S
    pool = {}
    for si, (w, h, D, cells, lo, hi) in enumerate(SERVED_SIZES):
        for mode in (0, 1, 2):
            for sl in range(2):
                spec = S.PairSpec(w, h, D, cells, lo, hi, 0.2 if mode == 2 else 0.0)
                pool[(si, mode, sl)] = tuple(_pinned(a) for a in
                                             S.make_pair(spec, S.SEED_BASE + 1000 + si * 10 + mode * 2 + sl)[:2])
    return pool


def _served_measure(slots: int, rates, requests: int, burst_n: int = 1000) -> dict:
    """The served stream: requests of four sizes and three modes with Poisson arrivals, through
    the served form (`slots` slots, continuous batching) and through the serial plain path
    (one slot) on the same arrival stream; plus a saturation burst for each."""
    import apg_sgm_b200 as apg
    pool = _served_pool()
    per_rate = max(1, requests // len(rates))
    # one warm server per form for the whole run: every (mode, size) has its engines resident
    # (the served form: one per slot) before the first timed request
    srv_served = _warm_server(apg, slots, pool)
    srv_serial = _warm_server(apg, 1, pool)
    results = []
    for k, rate in enumerate(rates):
        stream = _served_stream(per_rate, rate, 100 + k)
        served = _serve_stream(srv_served, pool, stream)
        serial = _serve_stream(srv_serial, pool, stream)
        results.append({"rate": rate, "requests": per_rate, "served": served, "serial": serial})
    burst = _served_stream(min(per_rate, burst_n), 0, 999)
    cap_served = _serve_stream(srv_served, pool, burst)
    cap_serial = _serve_stream(srv_serial, pool, burst)
    srv_served.close()
    srv_serial.close()
    # the GPU's own bound for this mix: the burst's pairs run one after another with inputs
    # already on the device (sum of single-pair device times)
    bucket_ms = _bucket_device_ms(apg, pool)
    burst_device_s = sum(bucket_ms[(si, mode)] for _, si, mode, _ in burst) / 1000.0
    return {"pool": pool, "per_rate": per_rate, "results": results, "burst": burst, "cap_served": cap_served,
            "cap_serial": cap_serial, "bucket_ms": bucket_ms, "device_bound": len(burst) / burst_device_s}


def run_served(args):
    rates = [float(r) for r in args.rates.split(",")]
    m = _served_measure(args.slots, rates, args.requests)
    cap_served, cap_serial, results, per_rate = m["cap_served"], m["cap_serial"], m["results"], m["per_rate"]
    bucket_ms, device_bound = m["bucket_ms"], m["device_bound"]
    mean_vox = float(np.mean([w * h * D for w, h, D, *_ in SERVED_SIZES]))
    top = results[-1]
    print(json.dumps({
        "metric": "served pairs/s with p50/p95/p99 latency (mixed sizes and modes, bit-exact)",
        "value": cap_served["pairs_per_s"], "unit": "pairs/s", "n_gpus": 1, "steps": per_rate * len(rates),
        "warmup": 4 * args.slots * len(SERVED_SIZES), "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16",
        "data": "synthetic",
        "config": {"workload": "served_mixed_stream", "sizes": "640x480 D64, 1242x375 D192, 1280x720 D128, "
                   "1920x1080 D256", "modes": "70% Balanced, 20% Fast, 10% HighQuality", "arrivals": "Poisson",
                   "rates": rates, "slots": args.slots, "hbm_budget_gb": 120, "pool_pairs": len(m["pool"])},
        "capacity": {"served_pairs_per_s": cap_served["pairs_per_s"], "serial_pairs_per_s": cap_serial["pairs_per_s"],
                     "speedup": cap_served["pairs_per_s"] / cap_serial["pairs_per_s"],
                     "served_voxels_per_s": cap_served["pairs_per_s"] * mean_vox, "burst_requests": len(m["burst"]),
                     "device_bound_pairs_per_s": device_bound,
                     "served_over_device_bound": cap_served["pairs_per_s"] / device_bound,
                     "bucket_device_ms": {f"{SERVED_SIZES[si][0]}x{SERVED_SIZES[si][1]} D{SERVED_SIZES[si][2]} "
                                          f"{MODE_NAMES[mo]}": round(v, 4) for (si, mo), v in sorted(bucket_ms.items())},
                     "served": cap_served, "serial": cap_serial},
        "rates": results,
        "latency_ms_at_top_rate": {"p50": top["served"]["p50_ms"], "p95": top["served"]["p95_ms"],
                                   "p99": top["served"]["p99_ms"]},
        "e2e": {"value": cap_served["pairs_per_s"], "unit": "pairs/s", "api": "apgcu_server_submit/wait (host buffers)"},
    }))


def systems_records(args) -> dict:
    """The two systems forms in brief, for the single-pair line: the 64-pair uneven batch (batched
    vs plain, same outputs) and a short served stream (served vs serial plain, p50/p95/p99)."""
    bm = _batched_measure(steps=3, warmup=2, clocks=False)
    batched = {"workload": "64 uneven Balanced pairs (24x 640x480 D64, 24x 1242x375 D192, 16x 1280x720 D128)",
               "steps": 3, "pairs_per_s": bm["npairs"] * 3 / (bm["batch_ms"] / 1000.0),
               "plain_pairs_per_s": bm["npairs"] * 3 / (bm["plain_ms"] / 1000.0),
               "speedup_vs_plain": bm["plain_ms"] / bm["batch_ms"], "identical_to_plain": bm["identical"],
               "ms_per_batch": bm["batch_ms"] / 3, "plain_ms_per_batch": bm["plain_ms"] / 3,
               "e2e_pairs_per_s": bm["npairs"] * bm["e2e_steps"] / bm["e2e_s"],
               "how": "device time of apgcu_batch_process_device against the same pairs as sequential "
                      "single-pair launches on one stream; inputs in HBM, L2 flushed between steps"}
    rate = 400.0
    sm = _served_measure(slots=4, rates=[rate], requests=args.served_requests, burst_n=args.served_requests)
    r = sm["results"][0]
    served = {"workload": "Poisson stream, sizes uniform over 640x480 D64 / 1242x375 D192 / 1280x720 D128 / "
                          "1920x1080 D256, modes 70% Balanced / 20% Fast / 10% HighQuality",
              "requests": sm["per_rate"], "offered_pairs_per_s": rate, "slots": 4,
              "pairs_per_s": r["served"]["pairs_per_s"],
              "p50_ms": r["served"]["p50_ms"], "p95_ms": r["served"]["p95_ms"], "p99_ms": r["served"]["p99_ms"],
              "serial": {"pairs_per_s": r["serial"]["pairs_per_s"], "p50_ms": r["serial"]["p50_ms"],
                         "p95_ms": r["serial"]["p95_ms"], "p99_ms": r["serial"]["p99_ms"]},
              "capacity_pairs_per_s": sm["cap_served"]["pairs_per_s"],
              "serial_capacity_pairs_per_s": sm["cap_serial"]["pairs_per_s"],
              "capacity_speedup": sm["cap_served"]["pairs_per_s"] / sm["cap_serial"]["pairs_per_s"],
              "device_bound_pairs_per_s": sm["device_bound"],
              "how": "latency from submission to outputs on the host (apgcu_server_submit / wait); capacity "
                     "from a saturation burst of the same mix; serial = the same server with one slot"}
    return {"batched": batched, "served": served}


def run_reference_batched(args):
    """The reference's Packed CPU path over the 64-pair batch, pair after pair; a step is one
    bounded sample: one pair of each size, scaled by the batch's pair counts."""
    from oracle import oracle as O
    from apg_sgm_b200 import synthetic as S
    specs = S.batched_mix()
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libapg_ref.so not built"}))
        return
    vox = sum(sp.width * sp.height * sp.max_disparity for sp in specs)
    sample = {i: S.make_pair(specs[i], S.SEED_BASE + i)[:2] for i in (0, 24, 48)}
    sess = {i: O.RefSession(O.config(1, specs[i].max_disparity, volume_backend=2)) for i in sample}
    weight = {0: 24, 24: 24, 48: 16}
    for _ in range(args.warmup):
        for i in sample:
            sess[i].process(*sample[i])
    total = 0.0
    for _ in range(args.steps):
        for i in sample:
            t0 = time.perf_counter()
            sess[i].process(*sample[i])
            total += (time.perf_counter() - t0) * weight[i]
    value = vox * args.steps / total
    print(json.dumps({
        "impl": "reference", "metric": "W*H*D/s, 64-pair uneven batch (Balanced, bit-exact)", "value": value,
        "unit": "voxels/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * total / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u16", "data": "synthetic", "config": {"workload": "batched_balanced_64_uneven", "pairs": 64},
        "cpu_baseline": {"value": value, "unit": "voxels/s", "cores": O.ref_threads(), "kind": "reference",
                         "sample": "per step one pair of each size, scaled by the pair counts"},
        "e2e": {"value": value, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def cpu_baseline(spec, mode, L, R, gpu_out, over=None):
    """Time the reference (Packed, all host cores) on pair 0 and check the GPU output against it."""
    from oracle import oracle as O
    over = over or {}
    vox = spec.width * spec.height * spec.max_disparity
    if O.ref_available():
        cfg = O.config(mode, spec.max_disparity, volume_backend=2, **over)
        sess = O.RefSession(cfg, bounded_reuse=True)
        for _ in range(2):
            ref = sess.process(L, R)
        ts = []
        for _ in range(5):
            t0 = time.perf_counter()
            ref = sess.process(L, R)
            ts.append(time.perf_counter() - t0)
        med = statistics.median(ts)
        dense_s = float("nan")
        if not over.get("hier_enable"):  # hierarchical mode rejects the Dense backend
            cfg_d = O.config(mode, spec.max_disparity, volume_backend=1)  # Auto==Dense for Fast/Balanced
            sd = O.RefSession(cfg_d, bounded_reuse=True)
            sd.process(L, R)
            t0 = time.perf_counter()
            sd.process(L, R)
            dense_s = time.perf_counter() - t0
        parity = all(np.array_equal(np.ascontiguousarray(gpu_out[k]).view(np.uint8),
                                    np.ascontiguousarray(ref[k]).view(np.uint8))
                     for k in ("disparity", "confidence", "invalid_reason", "reliable_mask"))
        return {"value": vox / med, "unit": "voxels/s", "cores": O.ref_threads(), "kind": "reference",
                "sample": f"pair 0 ({spec.width}x{spec.height} D{spec.max_disparity} {MODE_NAMES[mode]}), "
                          f"reference Packed backend, 2 warm-up + median of 5",
                "ms_per_pair": med * 1000, "dense_backend_ms_per_pair": dense_s * 1000,
                "stage_ms": ref["stage_ms"]}, parity
    cfg = O.config(mode, spec.max_disparity, **over)
    t0 = time.perf_counter()
    o = O.pipeline(cfg, L, R)
    dt = time.perf_counter() - t0
    parity = all(np.array_equal(np.ascontiguousarray(gpu_out[k]).view(np.uint8),
                                np.ascontiguousarray(o[k]).view(np.uint8))
                 for k in ("disparity", "confidence", "invalid_reason", "reliable_mask"))
    return {"value": vox / dt, "unit": "voxels/s", "cores": os.cpu_count(), "kind": "port",
            "sample": "pair 0, C oracle, 1 run"}, parity


def run_b200(args, wl):
    import torch
    import apg_sgm_b200 as apg
    from apg_sgm_b200 import replicas, synthetic as S

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    mode, spec_args, label, over = wl
    spec = S.PairSpec(*spec_args)
    w, h, D = spec.width, spec.height, spec.max_disparity
    # experimental scopes (ExperimentalSubpixelScope / ExperimentalInpaintScope) of this thread: every
    # frame below, device, e2e and Python binding alike, runs under them
    from apg_sgm_b200 import _lib as _scope_lib
    _scope_lib.lib().apgcu_set_experimental(*_scope_of(args))
    Dp = (D + 63) // 64 * 64
    npairs = 2
    # host images in page-locked memory: the end-to-end leg uploads them from there every step
    pairs = [tuple(_pinned(a) for a in S.make_pair(spec, S.SEED_BASE + rank * npairs + i)[:2]) for i in range(npairs)]
    cfg = apg.config_from_mode(mode, D, **over)
    eng = apg.Engine(cfg, device=local)
    tuning = [(k, int(v)) for k, v in (t.split("=", 1) for t in args.tune)]
    for k, v in tuning:
        eng.set_tuning(k, v)
    es = torch.cuda.ExternalStream(eng.stream, device=dev)
    d_in = [(torch.from_numpy(l).to(dev), torch.from_numpy(r).to(dev)) for l, r in pairs]
    d_disp = torch.empty((h, w), dtype=torch.float32, device=dev)
    d_conf = torch.empty((h, w), dtype=torch.float32, device=dev)
    d_reason = torch.empty((h, w), dtype=torch.uint8, device=dev)
    d_rel = torch.empty((h, w), dtype=torch.uint8, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()

    def step(i):
        l, r = d_in[i % npairs]
        eng.process_device(l.data_ptr(), r.data_ptr(), w, h, w, 1, d_disp.data_ptr(), d_conf.data_ptr(),
                           d_reason.data_ptr(), d_rel.data_ptr())

    for i in range(max(args.warmup, 3)):
        step(i)
    eng.sync()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    sampler.start()
    sampler.wait_first()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = apg.kernel_launch_count()
    sampler.mark("timed_start")
    with torch.cuda.stream(es):
        for k in range(args.steps):
            flush.zero_()  # L2 flush outside the timed step
            starts[k].record(es)
            step(k)
            ends[k].record(es)
    torch.cuda.synchronize()
    sampler.mark("timed_end")
    launches = apg.kernel_launch_count() - launches0

    # per-launch device times (a separate pass: the event after every launch is not in the timing)
    eng.set_debug(apg.DEBUG_PROFILE)
    per_kernel = {}
    with torch.cuda.stream(es):
        for k in range(min(args.steps, 20)):
            flush.zero_()
            step(k)
            for name, ms in eng.launch_profile():  # syncs on this step's last launch
                per_kernel.setdefault(name, []).append(ms)
    torch.cuda.synchronize()
    eng.set_debug(0)
    dev_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    if dist:
        dist.barrier()
    max_ms = replicas.max_over_ranks(dev_ms, dist, dev)  # the job's device time is the slowest rank's
    vox = w * h * D
    value = vox * args.steps * world / (max_ms / 1000.0)

    # end to end through the public C API (apg_session_process, src/c_api.cpp's entry point): host
    # images in, host result maps out, the copies inside every step
    import ctypes as C
    from apg_sgm_b200 import _lib
    lib = _lib.lib()
    opts = _lib.SessionOptions()
    opts.struct_size = C.sizeof(opts)
    opts.quality_mode, opts.memory_policy, opts.max_disparity, opts.backend = mode, 1, D, 3
    if over:
        # options the reference's C API does not carry: the full-configuration session
        sess_c = lib.apgcu_session_create_config(C.byref(cfg), 1, 0)
    else:
        sess_c = lib.apg_session_create_ex(C.byref(opts))
    for k, v in tuning:
        lib.apgcu_session_set_tuning(sess_c, k.encode(), v)
    res_c = lib.apg_result_create()
    views = [(_lib.ImageView(l.ctypes.data, w, h, w, 1), _lib.ImageView(r.ctypes.data, w, h, w, 1)) for l, r in pairs]
    rw, rh = C.c_int(), C.c_int()

    def e2e_step(i):
        lv, rv = views[i % npairs]
        rc = lib.apg_session_process(sess_c, C.byref(lv), C.byref(rv), res_c)
        if rc != 0:
            raise RuntimeError(lib.apg_session_get_last_error(sess_c).decode())
        return C.cast(lib.apg_result_get_disparity(res_c, C.byref(rw), C.byref(rh)), C.POINTER(C.c_float))[0]

    for i in range(max(args.warmup, 3)):
        e2e_step(i)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        e2e_step(k)
    e2e_s = time.perf_counter() - t0
    e2e_value = vox * args.steps * world / replicas.max_over_ranks(e2e_s, dist, dev)
    lib.apg_result_destroy(res_c)
    lib.apg_session_destroy(sess_c)

    # the same through the Python binding (StereoSession.process returns numpy views over a pooled
    # page-locked result block)
    sess = apg.StereoSession(mode=MODE_NAMES[mode].lower() if mode != 2 else "high_quality", max_disparity=D,
                             memory_policy="bounded_reuse", hierarchical=bool(over.get("hier_enable")))
    for k, v in tuning:
        sess.set_tuning(k, v)
    for i in range(max(args.warmup, 3)):
        sess.process(*pairs[i % npairs])
    npy = max(3, min(args.steps, 50))
    t0 = time.perf_counter()
    for k in range(npy):
        sess.process(*pairs[k % npairs])
    py_value = vox * npy / (time.perf_counter() - t0)
    clocks = sampler.stop()

    # dominant kernel and its roofline: the largest share of device time among the kernels with a
    # byte model (the HBM-bound ones); a latency-bound stage that outweighs it (the HighQuality
    # refiner's wavefront) is described beside it by its own model
    peak, peak_kind = _peaks()
    totals = {k: sum(v) for k, v in per_kernel.items() if k != "copy"}
    prof_total = sum(totals.values())
    vb = _volume_bytes(cfg, tuning)
    modelled = {k: v for k, v in totals.items()
                if _algorithmic_bytes(k, w, h, D, volume_source=True, npath=cfg.paths, vb=vb) > 0}
    top = max(modelled or totals, key=(modelled or totals).get)
    top_avg_ms = statistics.mean(per_kernel[top])
    alg = _algorithmic_bytes(top, w, h, D, volume_source=True, npath=cfg.paths, vb=vb)  # every mode's sweeps read a volume
    achieved = alg / (top_avg_ms / 1000.0) / 1e9
    roofline = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "volume_bytes_per_voxel": vb,
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": _profile_traffic(top, label), "algorithmic_bytes_per_launch": alg,
                "avg_launch_ms": top_avg_ms,
                "kernel_shares": {k: round(v / prof_total, 4) for k, v in sorted(totals.items(), key=lambda x: -x[1])},
                "kernel_avg_ms": {k: round(statistics.mean(per_kernel[k]), 5) for k in totals}}
    # the HBM-bound kernels (the SGM sweeps and the vertical aggregation) against the measured peak,
    # whichever kernel dominates; the cost kernels compute LUT costs and are issue-bound
    roofline["hbm_frac_by_kernel"] = {
        k: round(_algorithmic_bytes(k, w, h, D, volume_source=True, npath=cfg.paths, vb=vb) /
                 (statistics.mean(per_kernel[k]) / 1000.0) / 1e9 / peak, 4)
        for k in ("sgm_first", "sgm_fold5", "sgm_last_wta", "crossV") if k in per_kernel}
    if top in ("cost", "cost+crossH"):
        roofline["note"] = ("issue-bound: integer and LUT work per voxel (ncu issue active ~73%, DRAM ~8%); "
                            "the HBM fraction of its 2 B/voxel output is shown for reference")
    if "refine" in per_kernel:
        # the refiner: passes x a wavefront over the frame; a pixel's update needs its left and up
        # neighbours' values of the same pass, so a pass takes at least w + h - 1 dependent steps.
        # Work unit per pixel and pass: its 32-byte record, its packed left pixel (8 B), two packed
        # right-window pixels (16 B) and its value (4 B) = 60 B
        ref_ms = statistics.mean(per_kernel["refine"])
        passes = max(1, int(cfg.refine_iterations))
        steps_min = w + h - 1
        ref_bytes = 60.0 * w * h * passes
        roofline["latency_bound"] = {
            "kernel": "refine (HighQuality refiner: prep, band wavefront, draw indices)",
            "ms_per_frame": ref_ms, "share": round(totals["refine"] / prof_total, 4), "passes": passes,
            "min_dependent_steps_per_pass": steps_min,
            "ns_per_dependent_step": ref_ms * 1e6 / passes / steps_min,
            "algorithmic_bytes": ref_bytes,
            "hbm_frac": round(ref_bytes / (ref_ms / 1000.0) / 1e9 / peak, 4),
            "model": "each pass is a wavefront of at least w + h - 1 dependent steps (a pixel needs its "
                     "left and up neighbours of the same pass); time = passes x steps x step latency, so "
                     "ns_per_dependent_step is the figure to lower, the HBM fraction stays small by design"}

    out = {
        "metric": metric_name(mode, w, h, D, over), "value": value, "unit": "voxels/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": {"workload": label, "mode": MODE_NAMES[mode], "width": w, "height": h, "max_disparity": D,
                   "pairs_per_step": 1, "distinct_pairs": npairs, "l2": "flushed between steps (256 MiB write)",
                   "parallelism": f"replicas x{world}", **_scope_label(args),
                   **({"tuning": dict(tuning)} if tuning else {})},
        "e2e": {"value": e2e_value, "unit": "voxels/s", "h2d_bytes_per_step": 2 * w * h,
                "d2h_bytes_per_step": w * h * 10 + 64, "api": "apg_session_process (C API, BoundedReuse)" + (
                    "; session from apgcu_session_create_config" if over else ""),
                "python_binding_value": py_value},
        "gpu_launches": launches,
        "roofline": roofline,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        gpu0 = eng.process(*pairs[0])
        from oracle import oracle as O
        if O.ref_available():
            O.set_experimental(*_scope_of(args), reference=True)
        O.set_experimental(*_scope_of(args))
        cb, parity = cpu_baseline(spec, mode, pairs[0][0], pairs[0][1], gpu0, over)
        out["cpu_baseline"] = cb
        out["parity_vs_cpu_baseline"] = "bit-exact" if parity else "MISMATCH"
    del sess
    eng.close()
    if rank == 0 and world == 1 and args.systems:
        out.update(systems_records(args))
    if rank == 0:
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _batched_measure(steps: int, warmup: int, local: int = 0, dist=None, rank: int = 0, world: int = 1,
                     clocks: bool = True) -> dict:
    """The 64-pair uneven Balanced batch (24x 640x480 D64, 24x 1242x375 D192, 16x 1280x720 D128)
    through the batched form, against the same 64 pairs as sequential plain launches on one
    stream.  A step is the whole batch; inputs resident in HBM, L2 flushed between steps."""
    import torch
    import apg_sgm_b200 as apg
    from apg_sgm_b200 import _lib, replicas, synthetic as S

    dev = torch.device("cuda", local)
    specs = S.batched_mix()
    host = [tuple(_pinned(a) for a in S.make_pair(sp, S.SEED_BASE + rank * len(specs) + i)[:2])
            for i, sp in enumerate(specs)]
    vox = sum(sp.width * sp.height * sp.max_disparity for sp in specs)
    npairs = len(specs)
    d_in = [(torch.from_numpy(l).to(dev), torch.from_numpy(r).to(dev)) for l, r in host]

    def outs():
        return [{"disparity": torch.empty((sp.height, sp.width), dtype=torch.float32, device=dev),
                 "confidence": torch.empty((sp.height, sp.width), dtype=torch.float32, device=dev),
                 "invalid_reason": torch.empty((sp.height, sp.width), dtype=torch.uint8, device=dev),
                 "reliable_mask": torch.empty((sp.height, sp.width), dtype=torch.uint8, device=dev)}
                for sp in specs]

    o_plain, o_batch = outs(), outs()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    cfg = apg.config_from_mode(1, 128)
    # plain: one engine per size, all on one stream, the pairs one after another
    stream = torch.cuda.Stream(device=dev)
    engines = {}
    for sp in specs:
        if sp.max_disparity not in engines:
            engines[sp.max_disparity] = apg.Engine(apg.config_from_mode(1, sp.max_disparity), device=local,
                                                   stream=stream.cuda_stream)

    def plain_step():
        for sp, (l, r), o in zip(specs, d_in, o_plain):
            engines[sp.max_disparity].process_device(l.data_ptr(), r.data_ptr(), sp.width, sp.height, sp.width, 1,
                                                     o["disparity"].data_ptr(), o["confidence"].data_ptr(),
                                                     o["invalid_reason"].data_ptr(), o["reliable_mask"].data_ptr())

    batch = apg.Batch(cfg, device=local)
    recs = [_lib.Pair(l.data_ptr(), r.data_ptr(), sp.width, sp.height, sp.width, 1, sp.max_disparity,
                      o["disparity"].data_ptr(), o["confidence"].data_ptr(), o["invalid_reason"].data_ptr(),
                      o["reliable_mask"].data_ptr()) for sp, (l, r), o in zip(specs, d_in, o_batch)]

    # warm-up (the batched form tunes and captures its graphs here)
    for _ in range(max(warmup, 3)):
        with torch.cuda.stream(stream):
            plain_step()
        stream.synchronize()
        batch.process_device(recs)
    torch.cuda.synchronize()
    identical = all(torch.equal(a[k].view(torch.uint8), b[k].view(torch.uint8))
                    for a, b in zip(o_plain, o_batch) for k in a)

    # plain, timed on its stream
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            ev[k][0].record(stream)
            plain_step()
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    plain_ms = sum(a.elapsed_time(b) for a, b in ev)

    # batched: device time of every call (start event to the latest bucket end)
    sampler = ClockSampler(local) if clocks else None
    if sampler:
        sampler.start()
        sampler.wait_first()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = apg.kernel_launch_count()
    batch_ms = 0.0
    if sampler:
        sampler.mark("timed_start")
    for k in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        batch.process_device(recs)
        batch_ms += batch.last_time_ms
    torch.cuda.synchronize()
    if sampler:
        sampler.mark("timed_end")
    launches = apg.kernel_launch_count() - launches0
    clk = sampler.stop() if sampler else None
    batch_ms = replicas.max_over_ranks(batch_ms, dist, dev)
    plain_ms = replicas.max_over_ranks(plain_ms, dist, dev)

    # end to end: host images in, host maps out, through apgcu_batch_process
    e2e_steps = max(3, min(steps, 20))
    h_out = [{k: _pinned(np.zeros((sp.height, sp.width), dt)) for k, dt in
              (("disparity", np.float32), ("confidence", np.float32), ("invalid_reason", np.uint8),
               ("reliable_mask", np.uint8))} for sp in specs]
    for _ in range(2):
        batch.process([(l, r, sp.max_disparity) for sp, (l, r) in zip(specs, host)], out=h_out)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        batch.process([(l, r, sp.max_disparity) for sp, (l, r) in zip(specs, host)], out=h_out)
    e2e_s = time.perf_counter() - t0
    batch.close()
    for e in engines.values():
        e.close()
    return {"specs": specs, "host": host, "vox": vox, "npairs": npairs, "batch_ms": batch_ms, "plain_ms": plain_ms,
            "identical": bool(identical), "launches": launches, "clocks": clk, "e2e_s": e2e_s,
            "e2e_steps": e2e_steps}


def run_batched(args):
    """The 64-pair uneven batch as its own bench line (see _batched_measure)."""
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(torch.device("cuda", local))
    m = _batched_measure(args.steps, args.warmup, local, dist, rank, world)
    specs, host, vox, npairs = m["specs"], m["host"], m["vox"], m["npairs"]
    batch_ms, plain_ms = m["batch_ms"], m["plain_ms"]
    value = vox * args.steps * world / (batch_ms / 1000.0)
    plain_value = vox * args.steps * world / (plain_ms / 1000.0)
    e2e_value = vox * m["e2e_steps"] * world / m["e2e_s"]
    h2d = sum(2 * sp.width * sp.height for sp in specs)
    d2h = sum(10 * sp.width * sp.height for sp in specs)
    peak, peak_kind = _peaks()
    # the whole pipeline against the stage-boundary byte model (36 B per voxel for Balanced)
    achieved = 36.0 * vox / (batch_ms / args.steps / 1000.0) / 1e9
    out = {
        "metric": "W*H*D/s, 64-pair uneven batch (Balanced, bit-exact)", "value": value, "unit": "voxels/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": batch_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": {"workload": "batched_balanced_64_uneven", "pairs": npairs,
                   "sizes": "24x 640x480 D64, 24x 1242x375 D192, 16x 1280x720 D128", "voxels_per_step": vox,
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}"},
        "pairs_per_s": npairs * args.steps * world / (batch_ms / 1000.0),
        "plain": {"value": plain_value, "ms_per_step": plain_ms / args.steps,
                  "pairs_per_s": npairs * args.steps * world / (plain_ms / 1000.0),
                  "how": "the 64 pairs as sequential single-pair launches on one stream"},
        "speedup_vs_plain": plain_ms / batch_ms,
        "identical_to_plain": m["identical"],
        "e2e": {"value": e2e_value, "unit": "voxels/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "api": "apgcu_batch_process (host buffers)"},
        "gpu_launches": m["launches"],
        "roofline": {"bound": "hbm", "kernel": "pipeline (36 B/voxel stage-boundary model)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None},
        "clocks": m["clocks"],
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        if O.ref_available():
            # the reference on one pair of each size, scaled to the batch by pair counts
            tot = 0.0
            for i in (0, 24, 48):
                sp = specs[i]
                sess = O.RefSession(O.config(1, sp.max_disparity, volume_backend=2))
                sess.process(*host[i])
                t0 = time.perf_counter()
                sess.process(*host[i])
                tot += (time.perf_counter() - t0) * {0: 24, 24: 24, 48: 16}[i]
            out["cpu_baseline"] = {"value": vox / tot, "unit": "voxels/s", "cores": O.ref_threads(),
                                   "kind": "reference",
                                   "sample": "one pair of each size through the reference Packed backend, "
                                             "scaled by the batch's pair counts"}
    if rank == 0:
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


METRICS_SPEC = (1920, 1080, 256, 16, 0, 240, 0.2)
METRICS_BYTES_PER_PIXEL = 22  # est 4 + gt 4 + ranges 2+2 + refine maps 4+4 + visibility 1 + left image 1


def _metrics_inputs(seed: int):
    """A 1920x1080 evaluation frame: synthetic ground truth (on a 1/256 grid), an estimate with
    sub-pixel noise, gross errors and invalid pixels, refine maps, per-pixel ranges, the
    matchability mask as visibility and the left image."""
    from apg_sgm_b200 import synthetic as S
    spec = S.PairSpec(*METRICS_SPEC)
    L, _, gt = S.make_pair(spec, seed)
    rng = np.random.default_rng(seed)
    h, w = gt.shape
    gt = (np.round(gt.astype(np.float64) * 256) / 256).astype(np.float32)
    noise = (np.round(rng.normal(0, 0.7, (h, w)) * 65536) / 65536).astype(np.float32)
    gross = rng.random((h, w)) < 0.05
    noise[gross] += rng.integers(-20, 20, gross.sum()).astype(np.float32)
    est = (gt + noise).astype(np.float32)
    est[rng.random((h, w)) < 0.06] = -1.0
    before = (gt + 1.5 * noise).astype(np.float32)
    after = (gt + 1.1 * noise).astype(np.float32)
    r = rng.integers(2, 12, (h, w))
    rmin = (np.floor(gt) - r).astype(np.int16)
    rmax = (np.floor(gt) + r).astype(np.int16)
    vis = np.where(np.arange(w)[None, :] - np.round(gt) >= 0, 255, 0).astype(np.uint8)
    return {"est": est, "gt": gt, "rmin": rmin, "rmax": rmax, "before": before, "after": after, "vis": vis,
            "left": L}


def _metrics_call(fn, d):
    return fn(d["est"], d["gt"], (d["rmin"], d["rmax"]), d["before"], d["after"], d["vis"], 1e5, d["left"])


def run_metrics(args):
    """evaluate_stereo (src/metrics.cpp:119-502) over one 1920x1080 frame with every optional input.
    value: pixels/s with the inputs resident in HBM (L2 flushed between steps); e2e: the same call
    on page-locked host arrays (copies inside)."""
    import torch
    import apg_sgm_b200 as apg
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    host = {k: _pinned(v) for k, v in _metrics_inputs(11).items()}
    h, w = host["gt"].shape
    n = w * h
    d = {k: torch.from_numpy(v).to(dev) for k, v in host.items()}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    s = torch.cuda.Stream(device=dev)
    call = lambda arrs: _metrics_call(lambda *a: apg.evaluate_stereo(*a, stream=s.cuda_stream), arrs)  # noqa: E731
    torch.cuda.synchronize()
    for _ in range(max(args.warmup, 3)):
        call(d)
    # device time: CUDA events the library records on the launching stream around its two kernels
    # (a call's host work -- argument checks, the stream-ordered allocation, the 728-byte tally
    # copy and the synchronisation -- is outside them; e2e below includes everything)
    from apg_sgm_b200 import _lib
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    sampler.start()
    sampler.wait_first()
    launches0 = apg.kernel_launch_count()
    times = []
    sampler.mark("timed_start")
    with torch.cuda.stream(s):
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(s)
            m = call(d)
            ends[k].record(s)
            times.append(float(_lib.lib().apgcu_metrics_last_kernel_ms()))
    torch.cuda.synchronize()
    sampler.mark("timed_end")
    launches = apg.kernel_launch_count() - launches0
    clocks = sampler.stop()
    call_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    dev_ms = sum(times)
    value = n * args.steps / (dev_ms / 1000.0)
    # e2e: host arrays, copies inside the call
    for _ in range(3):
        _metrics_call(apg.evaluate_stereo, host)
    t0 = time.perf_counter()
    ne = max(3, min(args.steps, 50))
    for _ in range(ne):
        _metrics_call(apg.evaluate_stereo, host)
    e2e_s = (time.perf_counter() - t0) / ne
    peak, peak_kind = _peaks()
    alg = METRICS_BYTES_PER_PIXEL * n
    med_ms = statistics.mean(times)
    achieved = alg / (med_ms / 1000.0) / 1e9
    out = {
        "metric": f"evaluate_stereo pixels/s at {w}x{h} (every optional input)", "value": value, "unit": "pixels/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "metrics_1920x1080", "width": w, "height": h,
                   "inputs": "est, gt, ranges, refine before/after, visibility, left image",
                   "l2": "flushed between steps (256 MiB write)"},
        "e2e": {"value": n / e2e_s, "unit": "pixels/s", "h2d_bytes_per_step": alg,
                "d2h_bytes_per_step": (76 + 15) * 8, "api": "apgcu_evaluate_stereo, page-locked host arrays"},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": "metrics_kernel (+ final reduce, tally copy)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": None, "algorithmic_bytes_per_launch": alg, "avg_launch_ms": med_ms,
                     "note": "the two kernels per call (tally pass + fixed-order partial sum), library events",
                     "call_ms_median": statistics.median(call_ms)},
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        if O.ref_available():
            ref = lambda *a: O.evaluate_stereo(*a, reference=True)  # noqa: E731
            want = _metrics_call(ref, host)
            ts = []
            for _ in range(5):
                t0 = time.perf_counter()
                _metrics_call(ref, host)
                ts.append(time.perf_counter() - t0)
            med = statistics.median(ts)
            same = all(getattr(m, k) == getattr(want, k) for k, _ in m._fields_ if not k.startswith("reg_"))
            out["cpu_baseline"] = {"value": n / med, "unit": "pixels/s", "cores": 1, "kind": "reference",
                                   "sample": f"one {w}x{h} frame through the reference's evaluate_stereo, median of 5",
                                   "ms_per_frame": med * 1000}
            out["parity_vs_cpu_baseline"] = "identical record" if same else "MISMATCH"
    print(json.dumps(out))


def run_reference_metrics(args):
    """The reference's evaluate_stereo on the host for the metrics workload."""
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libapg_ref.so not built"}))
        return
    host = _metrics_inputs(11)
    h, w = host["gt"].shape
    ref = lambda *a: O.evaluate_stereo(*a, reference=True)  # noqa: E731
    for _ in range(args.warmup):
        _metrics_call(ref, host)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        _metrics_call(ref, host)
    total = time.perf_counter() - t0
    value = w * h * args.steps / total
    print(json.dumps({
        "impl": "reference", "metric": f"evaluate_stereo pixels/s at {w}x{h} (every optional input)", "value": value,
        "unit": "pixels/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * total / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": {"workload": "metrics_1920x1080", "width": w, "height": h},
        "cpu_baseline": {"value": value, "unit": "pixels/s", "cores": 1, "kind": "reference",
                         "sample": f"{args.steps} frames through the reference's evaluate_stereo (single-threaded)"},
        "e2e": {"value": value, "unit": "pixels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


FILES_SPEC = (1280, 720, 128, 12, 0, 120, 0.0)


def _write_file_pairs(apg, n: int, d):
    """n Balanced 1280x720 D128 pairs as binary PGM files in directory d (synthetic, seeded)."""
    from apg_sgm_b200 import synthetic as S
    spec = S.PairSpec(*FILES_SPEC)
    paths = []
    for i in range(n):
        L, R, _ = S.make_pair(spec, S.SEED_BASE + i)
        lp, rp = os.path.join(d, f"l{i:03d}.pgm"), os.path.join(d, f"r{i:03d}.pgm")
        apg.save_pgm(lp, L)
        apg.save_pgm(rp, R)
        paths.append((lp, rp))
    return paths


def run_files(args):
    """Pairs served from PGM files: the page-locked Loader reading ahead into the served form
    (serve_files) against the serial path (load_image, then one engine call per pair).  A step is
    the whole set of 48 pairs, files in the page cache; host time from the first read to the last
    result on the host."""
    import tempfile
    import torch
    import apg_sgm_b200 as apg
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    n = 48
    w, h, D = FILES_SPEC[0], FILES_SPEC[1], FILES_SPEC[2]
    with tempfile.TemporaryDirectory() as d:
        paths = _write_file_pairs(apg, n, d)
        srv = apg.Server(device=local, slots=4)
        srv.reserve(w, h, mode=1, max_disparity=D, count=4)
        depth = 16
        pool = [{k: _pinned(np.zeros((h, w), dt)) for k, dt in (("disparity", np.float32), ("confidence", np.float32),
                                                                  ("invalid_reason", np.uint8),
                                                                  ("reliable_mask", np.uint8))} for _ in range(depth)]
        ld = apg.Loader(threads=4)
        eng = apg.Engine(apg.config_from_mode(1, D), device=local)

        def served():
            for _ in apg.serve_files(srv, paths, mode=1, max_disparity=D, loader=ld, depth=depth, out_pool=pool):
                pass

        def serial():
            for lp, rp in paths:
                eng.process(apg.load_image(lp), apg.load_image(rp))

        for _ in range(max(args.warmup, 3) if args.warmup else 1):
            served()
            serial()
        launches0 = apg.kernel_launch_count()
        t0 = time.perf_counter()
        steps = max(1, min(args.steps, 5))
        for _ in range(steps):
            served()
        t_served = (time.perf_counter() - t0) / steps
        launches = apg.kernel_launch_count() - launches0
        t0 = time.perf_counter()
        for _ in range(steps):
            serial()
        t_serial = (time.perf_counter() - t0) / steps
        out = {
            "metric": f"pairs/s from PGM files, {w}x{h} D={D} Balanced", "value": n / t_served, "unit": "pairs/s",
            "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": t_served * 1000,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
            "config": {"workload": "files_48x_balanced_1280x720_d128", "pairs_per_step": n,
                       "loader_threads": 4, "server_slots": 4, "depth": depth,
                       "files": "binary PGM in the page cache"},
            "e2e": {"value": n / t_served, "unit": "pairs/s", "h2d_bytes_per_step": n * 2 * w * h,
                    "d2h_bytes_per_step": n * w * h * 10, "api": "serve_files (Loader -> Server, page-locked)"},
            "serial_value": n / t_serial, "served_over_serial": t_serial / t_served,
            "gpu_launches": launches,
            "loader_pinned_bytes": ld.pinned_bytes,
        }
        if not args.no_cpu_baseline:
            from oracle import oracle as O
            if O.ref_available():
                sess = O.RefSession(O.config(1, D, volume_backend=2), bounded_reuse=True)
                sample = paths[:4]
                for lp, rp in sample[:1]:
                    sess.process(O.ref_load_image(lp)[1], O.ref_load_image(rp)[1])
                t0 = time.perf_counter()
                for lp, rp in sample:
                    sess.process(O.ref_load_image(lp)[1], O.ref_load_image(rp)[1])
                tr = (time.perf_counter() - t0) / len(sample)
                out["cpu_baseline"] = {"value": 1.0 / tr, "unit": "pairs/s", "cores": O.ref_threads(),
                                       "kind": "reference",
                                       "sample": "4 of the file pairs: the reference's load_image + StereoSession "
                                                 "(Packed backend), all host threads"}
        ld.close()
        eng.close()
        srv.close()
        print(json.dumps(out))


def run_reference_files(args):
    """The reference's load_image + StereoSession over a bounded sample of the file pairs."""
    import tempfile
    import apg_sgm_b200 as apg  # only to write the input files
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libapg_ref.so not built"}))
        return
    D = FILES_SPEC[2]
    with tempfile.TemporaryDirectory() as d:
        paths = _write_file_pairs(apg, 4, d)
        sess = O.RefSession(O.config(1, D, volume_backend=2), bounded_reuse=True)
        for _ in range(args.warmup):
            sess.process(O.ref_load_image(paths[0][0])[1], O.ref_load_image(paths[0][1])[1])
        t0 = time.perf_counter()
        for k in range(args.steps):
            lp, rp = paths[k % len(paths)]
            sess.process(O.ref_load_image(lp)[1], O.ref_load_image(rp)[1])
        total = time.perf_counter() - t0
    value = args.steps / total
    print(json.dumps({
        "impl": "reference", "metric": f"pairs/s from PGM files, {FILES_SPEC[0]}x{FILES_SPEC[1]} D={D} Balanced",
        "value": value, "unit": "pairs/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * total / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u16", "data": "synthetic", "config": {"workload": "files_48x_balanced_1280x720_d128"},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": O.ref_threads(), "kind": "reference",
                         "sample": f"{args.steps} file pairs through load_image + StereoSession (Packed)"},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["batched", "served", "metrics1080", "files720"],
                    default="fast720")
    ap.add_argument("--requests", type=int, default=10000, help="served: total requests over the rates")
    ap.add_argument("--rates", default="50,100,200,400,600", help="served: Poisson arrival rates, pairs/s")
    ap.add_argument("--slots", type=int, default=4, help="served: requests in flight")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--subpixel", default="legacy",
                    help="ExperimentalSubpixelScope for the single-pair workloads: legacy | curv_gate | conf_gate | "
                         "stabilized, optionally :PARAM")
    ap.add_argument("--inpaint", default="legacy",
                    help="ExperimentalInpaintScope for the single-pair workloads: legacy | shadow_reclass, optionally :GAP")
    ap.add_argument("--tune", action="append", default=[],
                    help="engine tuning KEY=VALUE for the single-pair workloads' engines and sessions (repeatable)")
    ap.add_argument("--no-systems", action="store_true",
                    help="leave the batched and served sub-records out of the default (single GPU) line")
    ap.add_argument("--served-requests", type=int, default=400,
                    help="requests of the default line's served stream (and of its saturation burst)")
    args = ap.parse_args()
    # the headline line (default workload, one GPU) carries the two systems forms in brief
    args.systems = args.workload == "fast720" and not args.no_systems and args.gpus == 1
    if args.workload == "served":
        if args.impl == "reference":
            if int(os.environ.get("RANK", "0")) == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the served form has no reference counterpart; "
                                  "the reference CPU path is timed by the batched and single-pair workloads"}))
            return
        if int(os.environ.get("RANK", "0")) == 0:
            run_served(args)
        return
    if args.workload == "files720":
        if int(os.environ.get("RANK", "0")) == 0:
            (run_reference_files if args.impl == "reference" else run_files)(args)
        return
    if args.workload == "metrics1080":
        if int(os.environ.get("RANK", "0")) == 0:
            (run_reference_metrics if args.impl == "reference" else run_metrics)(args)
        return
    if args.workload == "batched":
        if args.impl == "reference":
            if int(os.environ.get("RANK", "0")) == 0:
                run_reference_batched(args)
            return
        run_batched(args)
        return
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) == 0:
            run_reference(args, wl)
        return
    run_b200(args, wl)


if __name__ == "__main__":
    main()
