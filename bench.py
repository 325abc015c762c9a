#!/usr/bin/env python
"""Benchmark of the dense-stereo depth stage: SGM MDE/s (W·H·D disparity evaluations per second).

Workload (one step = one solve): the 13 MP plain pair — 4160x3120 12-bit luma (mapped to bytes with (v+8)>>4),
D = 256 planes (= disparities 0..255), tile 64, the reference's P1/P2 and cost weights, synthetic seeded inputs
(1/f texture, six planar disparity segments, warped other view, sigma 2 DN noise). A solve is BoxFilter3 of both
images, the matching-cost volume, both aggregation passes and WTA — DenseStereoPyramid's work for one layer.

  value: inputs resident in HBM, depth left in HBM; timed with CUDA events on the library's stream.
  e2e:   the same through the public API from pinned host buffers: H2D of both images and D2H of the depth map
         are inside the timed region.
  --impl reference: the CPU restatement of the reference path (oracle/) on this host's cores, on a row strip of the
         same workload (the reference is C#/.NET and cannot run here).
Multi-GPU (torchrun): independent replicas, one solve per rank per step, no collective in the data path; the time
is the max over ranks.
"""
import argparse
import ctypes
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

WORKLOADS = {  # name: (W, H, D, tile, bits, description)
    "pair13mp": (4160, 3120, 256, 64, 12, "plain 13 MP pair 4160x3120 u16 12-bit -> u8, D=256, 8 paths, tile 64, P1 1, P2 500 adaptive"),
    "pair3mp": (2080, 1560, 256, 64, 12, "plain 3 MP pair 2080x1560 u16 12-bit -> u8, D=256, 8 paths, tile 64, P1 1, P2 500 adaptive"),
    "capture10": (2080, 1560, 0, 64, 0, "batched capture: 2080x1560 reference + 10 module cameras (1-6 MP crops, focal 1.0-2.7x, "
                  "D_k in {64,96,128,192}), one layer summing all costs, grey u8"),
    "pair1mp": (1040, 780, 64, 64, 8, "plain pair 1040x780 u8, D=64, 8 paths, tile 64, P1 1, P2 500 adaptive"),
    "preview": (520, 390, 32, 64, 8, "preview pair 520x390 u8, D=32, 8 paths, tile 64"),
}
W_, H_, D_, TILE, BITS, DESC = WORKLOADS["pair13mp"]
# Algorithmic HBM bytes per disparity element (DE = one pixel x one plane) of a layer's aggregation, aggregates not kept:
# pass +1 reads the u8 raw volume (1) and writes the u16 aggregates (2); pass -1 reads both again (1 + 2).
BYTES_PER_DE_AGG = 6
# DRAM bytes (read + write) per DE of a layer's aggregation as built (the path-group chains: 4 launches per layer),
# from ncu dram__bytes_read.sum + dram__bytes_write.sum of the four k_chains launches of the 2080x1560 D=256 pair:
# 2.655 + 4.315 + 4.317 + 2.730 GB = 14.02 GB for 830.7 MDE. The split design trades these extra bytes (aggregates read
# and written by both path groups, raw costs read by each) for a critical path of W or H steps.
TRAFFIC_PER_DE_LAYER = 14.02e9 / (2080 * 1560 * 256)


def metric():
    if BITS == 0:
        return f"SGM MDE/s (W·H·D per second), {W_}x{H_} reference + 10 module cameras D={D_}, bit-exact"
    return f"SGM MDE/s (W·H·D per second), {W_}x{H_} pair D={D_}, bit-exact"


def args_():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="lux", choices=["lux", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--sgm", default="auto", choices=["auto", "split", "wave", "fused"],
                   help="aggregation form of the timed solves (auto: the autotuner's choice, timed on the first solve of the "
                        "shape; a fixed form for profiler runs, whose timings would mislead the tuner)")
    p.add_argument("--no-served", action="store_true",
                   help="leave out the served stream and the batched capture objects of the default line")
    p.add_argument("--serve", action="store_true",
                   help="the served mixed request stream (Poisson arrivals of preview pairs, 13 MP pairs and module captures) "
                        "through the request server, against the plain one-request-at-a-time path on the same arrivals")
    p.add_argument("--requests", type=int, default=400)
    p.add_argument("--rate", type=float, default=40.0,
                   help="mean arrivals per second of the served stream (40/s: below what one request at a time keeps up "
                        "with, about 53/s, so the latencies compare the serving forms, not a growing backlog)")
    p.add_argument("--slots", type=int, default=2,
                   help="worker contexts of the request server (2 measured best: 3 stretches large requests' tails)")
    p.add_argument("--sweep", action="store_true",
                   help="throughput with 1, 4, 16 and 64 module captures in flight through the request server")
    p.add_argument("--cache", action="store_true",
                   help="the depth image cache: Set of the 4160x3120 full depth into the 5216x3912 cache, Fetch at the export levels")
    p.add_argument("--stereo", action="store_true",
                   help="stereo-image formation after the ISP: ten 2080x1560 module images warped, YUV'd and stored as 8 bits, "
                        "and the 4160x3120 reference guide's 8-bit warp")
    p.add_argument("--census", action="store_true",
                   help="the opt-in census mode (census, Hamming, 8-path SGM, WTA + subpixel + left/right) on the workload's pair")
    p.add_argument("--census-capture", action="store_true",
                   help="the census mode over a capture of 10 pairs (2080x1560, D in 64..192) batched, against the pairs one by one")
    p.add_argument("--pyramid", action="store_true",
                   help="the reference's whole dense job for a capture: DenseStereoPyramid.Run (six L16 layers) on five "
                        "2080x1560 colour cameras, then the upsample to 4160x3120")
    p.add_argument("--pyramid-size", default="2080x1560",
                   help="WxH of the --pyramid cameras (the finest layer); a smaller size is for profiling captures")
    p.add_argument("--cpu-rows", type=int, default=130, help="rows of the CPU sample strip")
    p.add_argument("--workload", default="pair13mp", choices=sorted(WORKLOADS),
                   help="pair13mp is the benchmark; the smaller pairs are for profiling captures")
    a = p.parse_args()
    global W_, H_, D_, TILE, BITS, DESC
    W_, H_, D_, TILE, BITS, DESC = WORKLOADS[a.workload]
    return a


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "fallback": True}


class ClockSampler:
    """nvidia-smi samples during the timed region: SM clock, max clock, throttle reasons."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def l2_note():
    raw = W_ * H_ * D_
    big = "larger" if raw > 126e6 else "NOT larger"
    return f"inputs {big} than L2 ({raw / 1e9:.2f} GB cost volume, {2 * raw / 1e9:.2f} GB aggregates)"


def workload(seed=0):
    from lux_b200 import synth
    if BITS == 0:  # a batched module capture: the reference grid W_ x H_ and 10 other cameras
        from lux_b200 import api
        mc = synth.module_capture(W_, H_, seed=seed, tile=TILE)
        global D_
        D_ = len(api.DenseStereo.planes(mc.near, mc.far, mc.calibs, mc.params.plane_density, 8))  # the layer's n
        return mc
    return synth.rectified_pair(W_, H_, D_, seed=seed, bits=BITS, tile=TILE)


def cpu_sample(wl, rows, threads):
    """The oracle (CPU restatement) on a row strip of the workload: cost prepass on `threads` cores, serial SGM."""
    from oracle import oracle as O
    # a strip of the reference image; the other cameras stay whole (their geometry is their own)
    imgs = [np.ascontiguousarray(wl.images[0][:rows])] + [np.ascontiguousarray(im) for im in wl.images[1:]]
    t0 = time.perf_counter()
    filt = [O.box_filter3(im) for im in imgs]
    O.layer(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, threads=threads)
    dt = time.perf_counter() - t0
    de = W_ * rows * D_
    return de / dt / 1e6, dt, de


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    wl = workload(0)
    for _ in range(a.warmup):
        cpu_sample(wl, a.cpu_rows, threads)
    vals, tot_de, tot_t = [], 0, 0.0
    for _ in range(a.steps):
        v, dt, de = cpu_sample(wl, a.cpu_rows, threads)
        vals.append(v)
        tot_de += de
        tot_t += dt
    value = tot_de / tot_t / 1e6
    sample = f"{W_}x{a.cpu_rows} row strip of the {W_}x{H_} D={D_} pair per step (oracle port: box filter, cost on {threads} threads, serial SGM, WTA)"
    print(json.dumps({
        "impl": "reference", "metric": metric(), "value": value, "unit": "MDE/s", "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": tot_t / a.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8/u16", "data": "synthetic",
        "config": {"workload": DESC, "sample_rows": a.cpu_rows},
        "cpu_baseline": {"value": value, "unit": "MDE/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "MDE/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_lux(a):
    import torch
    import torch.distributed as dist
    from lux_b200 import _lib, api

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    wl = workload(seed=rank)
    ctx = api.Context(local)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(lib.lux_sgm_stream(ctx.handle), device=torch.device("cuda", local))
    dev_imgs = [torch.from_numpy(im).cuda() for im in wl.images]
    host_imgs = [torch.from_numpy(im).pin_memory() for im in wl.images]
    depth_host = torch.empty((H_, W_), dtype=torch.float32).pin_memory()
    torch.cuda.synchronize()

    infos = []

    def solve(imgs):
        L = api.DenseLayer.compute(imgs, wl.gray, wl.calibs, wl.near, wl.far, wl.params, prefilter=True, sgm=a.sgm, ctx=ctx)
        infos.append((L.gpu_ms_cost, L.gpu_ms_sgm, L.gpu_ms_wta, L.sgm_kernel))
        return L

    def step_value():
        solve(dev_imgs).close()

    samples = getattr(wl, "samples", None)
    if samples is not None:
        # the cameras' 12-bit samples cross as 2 bytes a pixel and become the reference's byte images on the GPU
        host_samples = [torch.from_numpy(sm.view(np.int16)).pin_memory() for sm in samples]
        e2e_imgs = [torch.empty((H_, W_, 4), dtype=torch.uint8, device=torch.device("cuda", local)) for _ in samples]
        h2d_bytes = sum(sm.nbytes for sm in samples)
    else:
        h2d_bytes = sum(im.nbytes for im in wl.images)

    def step_e2e():
        if samples is not None:
            for hs, di in zip(host_samples, e2e_imgs):
                api.image_from_grey16(hs, BITS, ctx=ctx, out=di)
            L = solve(e2e_imgs)
        else:
            L = solve(host_imgs)
        ctx.check(lib.lux_layer_read(L.handle, _lib.FIELD_DEPTH, depth_host.data_ptr(), depth_host.numel() * 4))
        L.close()

    def timed(fn, k):
        for _ in range(a.warmup):
            fn()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        del infos[:]
        n0 = api.kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        launches = api.kernel_launches() - n0
        if world > 1:
            dist.barrier()
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, launches, list(infos)

    with ClockSampler(local) as clk:
        ms_v, launches, inf_v = timed(step_value, a.steps)
    ms_e, _, _ = timed(step_e2e, a.steps)
    de = W_ * H_ * D_
    value = world * de * a.steps / (ms_v / 1e3) / 1e6
    e2e = world * de * a.steps / (ms_e / 1e3) / 1e6
    sgm_ms = statistics.mean(x[1] for x in inf_v)
    cost_ms = statistics.mean(x[0] for x in inf_v)
    wta_ms = statistics.mean(x[2] for x in inf_v)
    pk = peaks()
    # per layer: the algorithmic bytes of both passes over the device time of the layer's aggregation launches
    achieved = BYTES_PER_DE_AGG * de / (sgm_ms / 1e3) / 1e9
    out = {
        "metric": metric(), "value": value, "unit": "MDE/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms_v / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8 cost / u16 aggregation", "data": "synthetic (seeded 1/f texture, planar disparity, warped view)",
        "config": {"workload": DESC,
                   "parallelism": f"replicas x{world}", "l2": l2_note(),
                   "stages_ms": {"cost": cost_ms, "sgm_2_passes": sgm_ms, "wta": wta_ms},
                   "sgm_kernel": {0: "exact-replay", 1: "fused-wavefront", 2: "path-group-chains", 3: "lean-wavefront"}.get(
                       inf_v[0][3] if inf_v else -1)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk.get("hbm_gbs"), "unit": "GB/s",
                     "frac": achieved / pk.get("hbm_gbs"), "traffic": TRAFFIC_PER_DE_LAYER * de,
                     "kernel": "SGM aggregation of one layer (both passes; 4 chain launches, or 2 fused ones below 2 MP)",
                     "bytes_per_de": BYTES_PER_DE_AGG, "traffic_per_de": TRAFFIC_PER_DE_LAYER,
                     "traffic_source": "ncu dram__bytes_read+write of the four 2080x1560 D=256 k_chains launches, scaled by DE",
                     "peak_source": "fallback" if pk.get("fallback") else "MEASURED_PEAKS.json hbm_gbs (measured)"},
        "e2e": {"value": e2e, "unit": "MDE/s", "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": W_ * H_ * 4,
                "path": ("host uint16 12-bit samples -> lux_image_from_grey16 -> lux_sgm_layer -> depth read back"
                         if samples is not None else "host RGBA8 images -> lux_sgm_layer -> depth read back")},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if BITS == 0 and world == 1:
        # the plain comparator of the batched capture: the reference against each module camera alone, one
        # two-camera solve (its own planes, D_k) after the other, inputs on the device
        pairs = []
        for k in range(1, len(wl.images)):
            imgs_k = [dev_imgs[0], dev_imgs[k]]
            pairs.append((imgs_k, [wl.gray[0], wl.gray[k]], [wl.calibs[0], wl.calibs[k]]))
        n_k = [len(api.DenseStereo.planes(wl.near, wl.far, c, wl.params.plane_density, 8)) for _, _, c in pairs]

        def plain_step():
            for imgs_k, g_k, c_k in pairs:
                api.DenseLayer.compute(imgs_k, g_k, c_k, wl.near, wl.far, wl.params, prefilter=True, ctx=ctx).close()
        ms_p, _, _ = timed(plain_step, a.steps)
        de_p = sum(W_ * H_ * n for n in n_k)
        out["config"]["plain_pairs"] = {"solves": len(pairs), "planes": n_k, "ms_per_capture": ms_p / a.steps,
                                        "mde_per_s": de_p * a.steps / (ms_p / 1e3) / 1e6,
                                        "note": "ten 2-camera layers one after another (sum of W·H·D_k per second)"}
    if rank == 0 and world == 1 and BITS != 0 and not a.no_served:
        # the metric's second half: the served mixed stream against the plain path, and the batched capture against its
        # ten-pair comparator (inputs on the device; wall clock for the stream, CUDA events for the capture)
        out["served"] = serve_stream(a)
        out["capture"] = capture_batched_vs_plain(a)
        # the reference's whole dense job of a capture (six-layer pyramid + upsample) beside its CPU port
        out["pyramid"] = pyramid_job(a, 2080, 1560, steps=5, warmup=3, cpu=not a.no_cpu_baseline)
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, dt, de_s = cpu_sample(wl, a.cpu_rows, threads)
        out["cpu_baseline"] = {"value": v, "unit": "MDE/s", "cores": threads, "kind": "port",
                               "sample": f"{W_}x{a.cpu_rows} row strip of the same pair ({de_s / 1e6:.0f} MDE, {dt:.1f} s): "
                                         f"oracle port, cost on {threads} threads, serial SGM as the reference"}
    if rank == 0:
        print(json.dumps(out))
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def serve_stream(a):
    """The served mixed stream (one GPU): requests drawn 50 % preview pairs (520x390, D=32, u8), 35 % 13 MP pairs
    (4160x3120, D=128, 12-bit) and 15 % batched module captures (2080x1560 reference + 10 cameras), arriving as a seeded
    Poisson process. Inputs stay on the device (a pool of distinct seeded inputs per kind); each request ends with its
    depth map on the host. Served: the request server (admission against a 120 GB budget, `slots` worker streams).
    Plain: the same arrivals solved one at a time on one stream. Latency = completion - arrival. Returns the stats."""
    import threading
    import torch
    from lux_b200 import api, synth
    torch.cuda.set_device(0)
    rng = np.random.default_rng(2026)

    def dev(images):
        return [torch.from_numpy(np.ascontiguousarray(im)).cuda() for im in images]

    pool = {"preview": [], "pair13mp": [], "capture10": []}
    for k in range(2):
        wl = synth.rectified_pair(520, 390, 32, seed=100 + k, bits=8, tile=64)
        pool["preview"].append((dev(wl.images), wl.gray, wl.calibs, wl.near, wl.far, wl.params, 520 * 390 * 32))
    for k in range(2):
        wl = synth.rectified_pair(4160, 3120, 128, seed=200 + k, bits=12, tile=64)
        pool["pair13mp"].append((dev(wl.images), wl.gray, wl.calibs, wl.near, wl.far, wl.params, 4160 * 3120 * 128))
    mc = synth.module_capture(2080, 1560, seed=300, tile=64)
    n_mc = len(api.DenseStereo.planes(mc.near, mc.far, mc.calibs, mc.params.plane_density, 8))
    pool["capture10"].append((dev(mc.images), mc.gray, mc.calibs, mc.near, mc.far, mc.params, 2080 * 1560 * n_mc))
    torch.cuda.synchronize()
    kinds = rng.choice(["preview", "pair13mp", "capture10"], size=a.requests, p=[0.5, 0.35, 0.15])
    picks = [pool[k][rng.integers(len(pool[k]))] for k in kinds]
    arrivals = np.cumsum(rng.exponential(1.0 / a.rate, size=a.requests))
    arrivals -= arrivals[0]

    # warm-up: every input solved once (builds, pools, lazy module loading)
    ctx = api.Context(0)
    for kind in pool:
        for r in pool[kind]:
            L = api.DenseLayer.compute(r[0], *r[1:6], prefilter=True, ctx=ctx)
            L.close()

    def plain():
        lat, t0 = [], time.perf_counter()
        for i, r in enumerate(picks):
            wait = t0 + arrivals[i] - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            L = api.DenseLayer.compute(r[0], *r[1:6], prefilter=True, ctx=ctx)
            _ = L.Depth
            L.close()
            lat.append(time.perf_counter() - t0 - arrivals[i])
        return np.array(lat), time.perf_counter() - t0

    def served():
        srv = api.Server(0, hbm_budget_bytes=120 * 10**9, slots=a.slots)
        # the worker contexts' first solves (module loading) and the memory pool's growth to what concurrent requests
        # hold are not part of the stream: every input twice, submitted at once so the slots run them side by side
        warm = [srv.submit(r[0], *r[1:6]) for _ in range(2) for kind in pool for r in pool[kind]]
        for t in warm:
            srv.wait(t)
        tickets = [None] * len(picks)
        t0 = time.perf_counter()

        def feeder():
            for i, r in enumerate(picks):
                wait = t0 + arrivals[i] - time.perf_counter()
                if wait > 0:
                    time.sleep(wait)
                tickets[i] = (srv.submit(r[0], *r[1:6]), time.perf_counter() - t0)
        th = threading.Thread(target=feeder)
        th.start()
        lat = []
        for i in range(len(picks)):
            while tickets[i] is None:
                time.sleep(0.0002)
            t, sub = tickets[i]
            res = srv.wait(t)
            assert res.status == 0
            lat.append(sub + (res.queue_ms + res.run_ms) / 1e3 - arrivals[i])
        th.join()
        total = time.perf_counter() - t0
        srv.close()
        return np.array(lat), total

    lat_p, tot_p = plain()
    lat_s, tot_s = served()
    ctx.close()
    de = sum(r[6] for r in picks)
    mix = {k: int((kinds == k).sum()) for k in pool}

    def stats(lat, tot):
        return {"req_per_s": len(picks) / tot, "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "mde_per_s": de / tot / 1e6, "wall_s": tot}

    shapes = {"preview": (520, 390, 32), "pair13mp": (4160, 3120, 128), "capture10": (2080, 1560, n_mc)}
    # plain: the library's default (the autotuner's choice); served: the server's choice by size
    forms = {k: {"plain": api.SGM_FORM_NAMES.get(api.tuned_form(w, h, n, 64), "size rule"),
                 "served": "split" if w * h >= 2000000 else "fused"} for k, (w, h, n) in shapes.items()}
    return {"workload": f"{a.requests} Poisson arrivals at {a.rate}/s: {mix}", "slots": a.slots, "hbm_budget_gb": 120,
            "sgm_forms": forms, "served": stats(lat_s, tot_s), "plain": stats(lat_p, tot_p)}


def capture_batched_vs_plain(a, steps=5, warmup=3):
    """The batched module capture (2080x1560 reference + 10 module cameras fused at cost level into one layer, the
    reference's multi-view sum) against its plain comparator: the reference against each module camera alone, ten
    two-camera solves one after another. Inputs on the device; ms per capture on the library's stream."""
    import torch
    from lux_b200 import api, synth
    mc = synth.module_capture(2080, 1560, seed=0, tile=64)
    ctx = api.Context(0)
    stream = torch.cuda.ExternalStream(ctx.lib.lux_sgm_stream(ctx.handle), device=torch.device("cuda", 0))
    dev_imgs = [torch.from_numpy(np.ascontiguousarray(im)).cuda() for im in mc.images]
    torch.cuda.synchronize()
    n = len(api.DenseStereo.planes(mc.near, mc.far, mc.calibs, mc.params.plane_density, 8))
    pairs = [([dev_imgs[0], dev_imgs[k]], [mc.gray[0], mc.gray[k]], [mc.calibs[0], mc.calibs[k]]) for k in range(1, len(dev_imgs))]
    n_k = [len(api.DenseStereo.planes(mc.near, mc.far, c, mc.params.plane_density, 8)) for _, _, c in pairs]

    def batched(sgm="auto"):
        api.DenseLayer.compute(dev_imgs, mc.gray, mc.calibs, mc.near, mc.far, mc.params, prefilter=True, sgm=sgm,
                               ctx=ctx).close()

    def plain(sgm="auto"):
        for imgs_k, g_k, c_k in pairs:
            api.DenseLayer.compute(imgs_k, g_k, c_k, mc.near, mc.far, mc.params, prefilter=True, sgm=sgm, ctx=ctx).close()

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    ms_b, ms_p = timed(batched), timed(plain)
    # the size rule the autotuner replaces (path-group chains from about 2 MP, so every layer here): the same work
    ms_bf, ms_pf = timed(lambda: batched("split")), timed(lambda: plain("split"))
    form = api.SGM_FORM_NAMES.get(api.tuned_form(2080, 1560, n, mc.params.tile), "untuned")
    ctx.close()
    return {"workload": "2080x1560 reference + 10 module cameras (1-6 MP crops, focal 1.0-2.7x, D_k 64-192), u8",
            "batched": {"ms_per_capture": ms_b, "planes": n, "mde_per_s": 2080 * 1560 * n / ms_b / 1e3, "sgm": form,
                        "note": "one layer summing the ten cameras' costs (the reference's multi-view sum)"},
            "plain": {"ms_per_capture": ms_p, "planes": n_k, "mde_per_s": sum(2080 * 1560 * k for k in n_k) / ms_p / 1e3,
                      "note": "ten two-camera layers one after another"},
            "size_rule": {"batched_ms": ms_bf, "plain_ms": ms_pf,
                          "note": "the same two jobs with the aggregation form fixed by size (path-group chains), "
                                  "against the autotuned forms above"}}


def run_serve(a):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    st = serve_stream(a)
    out = {"metric": "served depth requests/s (mixed Poisson stream), with p50/p99 latency, served vs plain",
           "value": st["served"]["req_per_s"], "unit": "req/s", "n_gpus": 1, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u8 cost / u16 aggregation", "data": "synthetic (seeded pools per kind)",
           "config": {"workload": st["workload"], "slots": st["slots"], "hbm_budget_gb": st["hbm_budget_gb"],
                      "sgm_forms": st["sgm_forms"]},
           "served": st["served"], "plain": st["plain"]}
    print(json.dumps(out))


def run_sweep(a):
    """Saturation: N batched module captures (2080x1560 reference + 10 cameras, two distinct seeded inputs on the device)
    submitted at once to the request server, for N in 1, 4, 16, 64; MDE/s of the whole batch and its wall time."""
    import torch
    from lux_b200 import api, synth
    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(0)
    caps = []
    for k in range(2):
        mc = synth.module_capture(2080, 1560, seed=400 + k, tile=64)
        n = len(api.DenseStereo.planes(mc.near, mc.far, mc.calibs, mc.params.plane_density, 8))
        caps.append(([torch.from_numpy(np.ascontiguousarray(im)).cuda() for im in mc.images], mc, 2080 * 1560 * n))
    torch.cuda.synchronize()
    srv = api.Server(0, hbm_budget_bytes=120 * 10**9, slots=a.slots)
    for imgs, mc, _ in caps:  # warm-up
        srv.wait(srv.submit(imgs, mc.gray, mc.calibs, mc.near, mc.far, mc.params))
    points = []
    for n_flight in (1, 4, 16, 64):
        t0 = time.perf_counter()
        tickets = [srv.submit(caps[i % 2][0], caps[i % 2][1].gray, caps[i % 2][1].calibs, caps[i % 2][1].near,
                              caps[i % 2][1].far, caps[i % 2][1].params) for i in range(n_flight)]
        for t in tickets:
            assert srv.wait(t).status == 0
        dt = time.perf_counter() - t0
        de = sum(caps[i % 2][2] for i in range(n_flight))
        points.append({"in_flight": n_flight, "mde_per_s": de / dt / 1e6, "wall_s": dt})
    srv.close()
    print(json.dumps({"metric": "MDE/s with N module captures in flight (request server)", "value": points[-1]["mde_per_s"],
                      "unit": "MDE/s", "n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                      "dtype": "u8 cost / u16 aggregation", "data": "synthetic (two seeded captures on the device)",
                      "config": {"workload": "batched module capture 2080x1560 + 10 cameras", "slots": a.slots},
                      "sweep": points}))


# ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_depth_cache_set launch, 4160x3120 -> 5216x3912
SET_TRAFFIC = 52.01e6 + 28.92e6


def run_cache(a):
    """The depth image cache (DepthCache.cs:136-181) on one GPU. Set: the 4160x3120 full depth (the upsample's output)
    into the 5216x3912 cache of a 10432x7824 canvas (FromFullDepth); Fetch: the whole frame at pipeline levels 0 (the
    canvas, a 2x upsample of the cache) and 2 (2608x1956). value = cache pixels per second of Set with the depth in HBM,
    L2 flushed (a 256 MB write) before every timed launch; e2e = the same from a pinned host depth map to a pinned host
    cache. Roofline: Set reads each source pixel once and writes each cache pixel (4 + 4 bytes per pixel); traffic is
    ncu's dram__bytes_read.sum + dram__bytes_write.sum of one Set launch of this workload (writes still in L2 when the
    kernel ends are not counted)."""
    import torch
    from lux_b200 import api
    if int(os.environ.get("RANK", "0")) != 0:
        return
    w, h, cw, ch = 4160, 3120, 5216, 3912
    rng = np.random.default_rng(7)
    depth = np.exp(rng.uniform(np.log(400.0), np.log(2.0e5), (h, w))).astype(np.float32)
    pk = peaks()
    algo_set = 4 * (w * h + cw * ch)
    desc = f"depth cache Set {w}x{h} full depth -> {cw}x{ch} cache; Fetch at levels 0 (10432x7824) and 2 (2608x1956)"
    threads = 1
    if a.impl == "reference":
        from oracle import oracle as O
        for _ in range(a.warmup):
            O.depth_cache_set(depth, cw, ch)
        t0 = time.perf_counter()
        for _ in range(a.steps):
            O.depth_cache_set(depth, cw, ch)
        dt = (time.perf_counter() - t0) / a.steps
        v = cw * ch / dt / 1e6
        print(json.dumps({"impl": "reference", "metric": "depth cache Set Mpix/s (cache pixels per second), bit-exact",
                          "value": v, "unit": "Mpix/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
                          "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "f32", "data": "synthetic", "config": {"workload": desc},
                          "cpu_baseline": {"value": v, "unit": "Mpix/s", "cores": threads, "kind": "port",
                                           "sample": "the whole Set, oracle port (scalar C)"},
                          "e2e": {"value": v, "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    torch.cuda.set_device(0)
    ctx = api.Context(0)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(lib.lux_sgm_stream(ctx.handle), device=torch.device("cuda", 0))
    d_depth = torch.from_numpy(depth).cuda()
    d_cache = torch.empty((ch, cw), dtype=torch.float32, device="cuda")
    h_depth = torch.from_numpy(depth).pin_memory()
    h_cache = torch.empty((ch, cw), dtype=torch.float32).pin_memory()
    flush = torch.empty(64 * 2**20, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()

    def set_dev():
        ctx.check(lib.lux_depth_cache_set(ctx.handle, d_depth.data_ptr(), w, h, 1, cw, ch, d_cache.data_ptr(), 1))

    def set_host():
        ctx.check(lib.lux_depth_cache_set(ctx.handle, h_depth.data_ptr(), w, h, 0, cw, ch, h_cache.data_ptr(), 0))

    def timed(fn, k, flush_l2):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        total = 0.0
        n0 = api.kernel_launches()
        for _ in range(k):
            if flush_l2:
                with torch.cuda.stream(stream):
                    flush.fill_(1.0)
                    torch.cuda._sleep(200000)  # keeps the stream busy while the host reaches the launch: no idle gap timed
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            total += e0.elapsed_time(e1)
        return total / k, api.kernel_launches() - n0

    with ClockSampler(0) as clk:
        ms_set, launches = timed(set_dev, a.steps, True)
    ms_e2e, _ = timed(set_host, a.steps, False)
    fetch = {}
    for lv, dims in ((0, (10432, 7824)), (2, (2608, 1956))):
        out = torch.empty((dims[1], dims[0]), dtype=torch.float32, device="cuda")

        def fetch_dev():
            ctx.check(lib.lux_depth_cache_fetch(ctx.handle, d_cache.data_ptr(), cw, ch, 1, 0, 0, dims[0], dims[1], dims[0],
                                                dims[1], out.data_ptr(), 1))
        ms, _ = timed(fetch_dev, a.steps, True)
        # algorithmic bytes: every cache pixel the resample reads, once (all of them for level 0; a quarter for level 2),
        # plus the output
        read_px = cw * ch if lv == 0 else dims[0] * dims[1]
        gbs = 4 * (read_px + dims[0] * dims[1]) / (ms / 1e3) / 1e9
        fetch[f"level{lv}"] = {"dims": list(dims), "ms": ms, "mpix_per_s": dims[0] * dims[1] / (ms / 1e3) / 1e6, "gbs": gbs,
                               "frac": gbs / pk.get("hbm_gbs")}
    achieved = algo_set / (ms_set / 1e3) / 1e9
    out = {"metric": "depth cache Set Mpix/s (cache pixels per second), bit-exact", "value": cw * ch / (ms_set / 1e3) / 1e6,
           "unit": "Mpix/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_set,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (log-uniform depth 400 mm .. 200 m)",
           "config": {"workload": desc, "l2": "flushed (256 MB write) before every timed Set and Fetch"},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk.get("hbm_gbs"), "unit": "GB/s",
                        "frac": achieved / pk.get("hbm_gbs"), "traffic": SET_TRAFFIC, "kernel": "k_depth_cache_set",
                        "bytes_per_pixel": algo_set / (cw * ch),
                        "peak_source": "fallback" if pk.get("fallback") else "MEASURED_PEAKS.json hbm_gbs (measured)"},
           "e2e": {"value": cw * ch / (ms_e2e / 1e3) / 1e6, "unit": "Mpix/s", "h2d_bytes_per_step": 4 * w * h,
                   "d2h_bytes_per_step": 4 * cw * ch},
           "fetch": fetch, "gpu_launches": int(launches), "clocks": clk.summary()}
    if not a.no_cpu_baseline:
        from oracle import oracle as O
        t0 = time.perf_counter()
        for _ in range(3):
            O.depth_cache_set(depth, cw, ch)
        dt = (time.perf_counter() - t0) / 3
        out["cpu_baseline"] = {"value": cw * ch / dt / 1e6, "unit": "Mpix/s", "cores": 1, "kind": "port",
                               "sample": f"the whole Set ({dt:.2f} s), oracle port (scalar C), 3 runs"}
    print(json.dumps(out))
    ctx.close()


def run_stereo(a):
    """Stereo-image formation (StereoImageBuilder.Create after the ISP, StereoImage.cs) for a capture: ten module images,
    each a 2080x1560 half-resolution ISP output (float RGBA) warped through its own aligned calibration into the
    2080x1560 view, ConvertToYUV and the 8-bit store (the dense solve's inputs, left in HBM); plus the reference guide's
    8-bit warp of the 4160x3120 ISP'd reference image (ReferenceGuide.cs). value = stereo-image pixels per second with
    the ISP outputs in HBM (the 10 sources, 520 MB, exceed L2); e2e = the same from pinned host images to host 8-bit
    images. Roofline (HBM): per output pixel the 16-byte source pixel read once and the 4-byte result written."""
    import torch
    from lux_b200 import api, synth
    if int(os.environ.get("RANK", "0")) != 0:
        return
    sw, sh, n_img = 2080, 1560, 10
    srcs = [synth.isp_image(sw, sh, seed=k) for k in range(n_img)]
    acs = [synth.aligned_calib(sw, sh, sw, sh, seed=k, angle_deg=0.3 * (k - 5)) for k in range(n_img)]
    neutral = (0.5, 1.0, 0.6)
    gains = [1.0] + [0.9 + 0.02 * k for k in range(1, n_img)]
    guide_src = np.random.default_rng(3).integers(0, 256, (3120, 4160, 4), dtype=np.uint8)
    guide_ac = synth.aligned_calib(4160, 3120, 4160, 3120, seed=99, angle_deg=0.0)
    desc = (f"{n_img} stereo images {sw}x{sh} (float RGBA ISP output -> Lanczos-3 CRA warp -> YUV -> 8-bit) + the 4160x3120 "
            "reference guide 8-bit warp")
    pk = peaks()
    if a.impl == "reference":
        from oracle import oracle as O
        t0 = time.perf_counter()
        O.stereo_image(srcs[0], gains[0], sw, sh, acs[0], 2, neutral)
        dt = time.perf_counter() - t0
        v = sw * sh / dt / 1e6
        print(json.dumps({"impl": "reference", "metric": "stereo images Mpix/s (output pixels per second), bit-exact",
                          "value": v, "unit": "Mpix/s", "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": dt * 1e3 * n_img,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                          "config": {"workload": desc},
                          "cpu_baseline": {"value": v, "unit": "Mpix/s", "cores": 1, "kind": "port",
                                           "sample": "one 2080x1560 stereo image, oracle port (scalar C)"},
                          "e2e": {"value": v, "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    torch.cuda.set_device(0)
    ctx = api.Context(0)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(lib.lux_sgm_stream(ctx.handle), device=torch.device("cuda", 0))
    d_src = [torch.from_numpy(x).cuda() for x in srcs]
    h_src = [torch.from_numpy(x).pin_memory() for x in srcs]
    d_out = [torch.empty((sh, sw, 4), dtype=torch.uint8, device="cuda") for _ in range(n_img)]
    h_out = [torch.empty((sh, sw, 4), dtype=torch.uint8).pin_memory() for _ in range(n_img)]
    d_yuv = torch.empty((sh, sw, 4), dtype=torch.float32, device="cuda")
    d_gsrc = torch.from_numpy(guide_src).cuda()
    d_guide = torch.empty((3120, 4160, 4), dtype=torch.uint8, device="cuda")
    cac = [ac.to_c() for ac in acs]
    gac = guide_ac.to_c()
    nb = np.ascontiguousarray(np.asarray(neutral, np.float32))
    torch.cuda.synchronize()

    def step(on_dev):
        for k in range(n_img):
            src = d_src[k] if on_dev else h_src[k]
            out = d_out[k] if on_dev else h_out[k]
            yuv = d_yuv.data_ptr() if k == 0 else None  # the reference camera keeps its YUV floats (RefYuv)
            ctx.check(lib.lux_stereo_image(ctx.handle, src.data_ptr(), sw, sh, 1 if on_dev else 0, gains[k], ctypes.byref(cac[k][0]),
                                           sw, sh, 2, nb.ctypes.data, out.data_ptr(), 1 if on_dev else 0, yuv, 1))

    def guide():
        img = api.L.Img(d_gsrc.data_ptr(), 4160, 3120, 4160, 1)
        ctx.check(lib.lux_warp_rgba8(ctx.handle, ctypes.byref(img), ctypes.byref(gac[0]), 4160, 3120, d_guide.data_ptr(), 1))

    def timed(fn, k):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        n0 = api.kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k, api.kernel_launches() - n0

    with ClockSampler(0) as clk:
        ms_v, launches = timed(lambda: step(True), a.steps)
    ms_e, _ = timed(lambda: step(False), a.steps)
    ms_g, _ = timed(guide, a.steps)
    px = n_img * sw * sh
    algo = px * (16 + 4) + sw * sh * 16  # sources read once, 8-bit results, the reference camera's YUV floats
    achieved = algo / (ms_v / 1e3) / 1e9
    out = {"metric": "stereo images Mpix/s (output pixels per second), bit-exact", "value": px / (ms_v / 1e3) / 1e6,
           "unit": "Mpix/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_v, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (1/f texture ISP images, rotation + CRA calibrations)",
           "config": {"workload": desc, "l2": f"ten sources of {sw * sh * 16 / 1e6:.0f} MB each, 520 MB per step (larger than L2)"},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk.get("hbm_gbs"), "unit": "GB/s",
                        "frac": achieved / pk.get("hbm_gbs"), "traffic": None, "kernel": "k_warp_f32<1> (ten launches)",
                        "bytes_per_pixel": algo / px,
                        "peak_source": "fallback" if pk.get("fallback") else "MEASURED_PEAKS.json hbm_gbs (measured)"},
           "e2e": {"value": px / (ms_e / 1e3) / 1e6, "unit": "Mpix/s", "h2d_bytes_per_step": n_img * sw * sh * 16,
                   "d2h_bytes_per_step": n_img * sw * sh * 4},
           "guide": {"ms": ms_g, "mpix_per_s": 4160 * 3120 / (ms_g / 1e3) / 1e6},
           "gpu_launches": int(launches), "clocks": clk.summary()}
    if not a.no_cpu_baseline:
        from oracle import oracle as O
        t0 = time.perf_counter()
        O.stereo_image(srcs[0], gains[0], sw, sh, acs[0], 2, neutral)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": sw * sh / dt / 1e6, "unit": "Mpix/s", "cores": 1, "kind": "port",
                               "sample": f"one {sw}x{sh} stereo image ({dt:.1f} s), oracle port (scalar C)"}
    print(json.dumps(out))
    ctx.close()


def run_census(a):
    """The opt-in census stereo mode on the workload's pair (default: 4160x3120, D=256): value = W·H·D per second with the
    images in HBM and the disparities left there; e2e from host images to host disparities. Roofline (HBM), the
    aggregation's algorithmic bytes: the eight path launches each read the u8 cost volume once and read-modify-write the
    u16 path sums (the first only writes): 8·1 + 7·4 + 2 = 38 bytes per DE."""
    import torch
    from lux_b200 import _lib, api
    if int(os.environ.get("RANK", "0")) != 0:
        return
    D = D_
    wl = workload(0)
    left, right = wl.images[0], wl.images[1]
    if a.impl == "reference":
        from oracle import census_oracle as C
        rows = 48
        t0 = time.perf_counter()
        C.census_sgm(left[:rows, :, 0], right[:rows, :, 0], D, 10, 120)
        dt = time.perf_counter() - t0
        v = W_ * rows * D / dt / 1e6
        print(json.dumps({"impl": "reference", "metric": f"census SGM MDE/s, {W_}x{H_} pair D={D}", "value": v, "unit": "MDE/s",
                          "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "u8 cost / u16 aggregation", "data": "synthetic", "config": {"workload": DESC},
                          "cpu_baseline": {"value": v, "unit": "MDE/s", "cores": 1, "kind": "port",
                                           "sample": f"{W_}x{rows} strip, numpy restatement"},
                          "e2e": {"value": v, "unit": "MDE/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    torch.cuda.set_device(0)
    ctx = api.Context(0)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(lib.lux_sgm_stream(ctx.handle), device=torch.device("cuda", 0))
    d_imgs = [torch.from_numpy(im).cuda() for im in (left, right)]
    h_imgs = [torch.from_numpy(im).pin_memory() for im in (left, right)]
    d_out = torch.empty((H_, W_), dtype=torch.float32, device="cuda")
    h_out = torch.empty((H_, W_), dtype=torch.float32).pin_memory()
    prm = _lib.CensusParams(D, 10, 120, 1, 1, 1)
    torch.cuda.synchronize()

    def step(on_dev):
        src = d_imgs if on_dev else h_imgs
        il = _lib.Img(src[0].data_ptr(), W_, H_, W_, 1 if on_dev else 0)
        ir = _lib.Img(src[1].data_ptr(), W_, H_, W_, 1 if on_dev else 0)
        out = d_out if on_dev else h_out
        ctx.check(lib.lux_census_sgm(ctx.handle, ctypes.byref(il), ctypes.byref(ir), ctypes.byref(prm), out.data_ptr(),
                                     1 if on_dev else 0))

    def timed(fn, k):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        n0 = api.kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k, api.kernel_launches() - n0

    with ClockSampler(0) as clk:
        ms_v, launches = timed(lambda: step(True), a.steps)
    ms_e, _ = timed(lambda: step(False), a.steps)
    de = W_ * H_ * D
    pk = peaks()
    achieved = 38 * de / (ms_v / 1e3) / 1e9  # the whole step's time: an upper bound on the aggregation's
    out = {"metric": f"census SGM MDE/s (W·H·D per second), {W_}x{H_} pair D={D}, opt-in mode", "value": de / (ms_v / 1e3) / 1e6,
           "unit": "MDE/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_v, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "u8 cost / u16 aggregation", "data": "synthetic",
           "config": {"workload": DESC + " (census mode: 9x7 census, P1 10, P2 120, subpixel, left/right)", "l2": l2_note()},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk.get("hbm_gbs"), "unit": "GB/s", "frac": achieved / pk.get("hbm_gbs"),
                        "traffic": None, "kernel": "the whole census step (38 B/DE of aggregation over the step's time)",
                        "peak_source": "fallback" if pk.get("fallback") else "MEASURED_PEAKS.json hbm_gbs (measured)"},
           "e2e": {"value": de / (ms_e / 1e3) / 1e6, "unit": "MDE/s", "h2d_bytes_per_step": 2 * W_ * H_ * 4, "d2h_bytes_per_step": W_ * H_ * 4},
           "gpu_launches": int(launches), "clocks": clk.summary()}
    print(json.dumps(out))
    ctx.close()


def run_census_capture(a):
    """The census mode over one capture: 10 pairs on a 2080x1560 reference grid with D cycling 64, 96, 128, 192, images in
    HBM. Batched: one lux_census_capture (every stage one launch over all pairs, the reference's census once, then the
    fusion). Plain: ten lux_census_sgm solves one after another, then lux_fuse_disparities. value = Σ W·H·D_k per second
    of the batched form."""
    import torch
    from lux_b200 import _lib, api, synth
    if int(os.environ.get("RANK", "0")) != 0:
        return
    w, h = 2080, 1560
    ds = [(64, 96, 128, 192)[k % 4] for k in range(10)]
    ref, others, fb = synth.census_capture(w, h, ds, seed=11)
    torch.cuda.set_device(0)
    ctx = api.Context(0)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(lib.lux_sgm_stream(ctx.handle), device=torch.device("cuda", 0))
    rgba = lambda im: torch.from_numpy(np.repeat(im[..., None], 4, axis=2)).cuda()
    d_ref, d_oth = rgba(ref), [rgba(o) for o in others]
    img = lambda t: _lib.Img(t.data_ptr(), w, h, w, 1)
    c_ref = img(d_ref)
    c_oth = (_lib.Img * len(d_oth))(*[img(t) for t in d_oth])
    dsa = np.asarray(ds, np.int32)
    prm = _lib.CensusParams(0, 10, 120, 1, 1, 1)
    depth = torch.empty((h, w), dtype=torch.float32, device="cuda")
    disps = [torch.empty((h, w), dtype=torch.float32, device="cuda") for _ in ds]
    dptrs = (ctypes.c_void_p * len(ds))(*[t.data_ptr() for t in disps])
    torch.cuda.synchronize()

    def batched():
        ctx.check(lib.lux_census_capture(ctx.handle, len(ds), ctypes.byref(c_ref), c_oth, dsa.ctypes.data, fb.ctypes.data,
                                         ctypes.byref(prm), depth.data_ptr(), 1, None))

    def plain():
        for k, d in enumerate(ds):
            pk = _lib.CensusParams(d, 10, 120, 1, 1, 1)
            ctx.check(lib.lux_census_sgm(ctx.handle, ctypes.byref(c_ref), ctypes.byref(c_oth[k]), ctypes.byref(pk), disps[k].data_ptr(), 1))
        ctx.check(lib.lux_fuse_disparities(ctx.handle, dptrs, fb.ctypes.data, len(ds), w, h, 1, depth.data_ptr(), 1))

    def timed(fn, k):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        n0 = api.kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k, (api.kernel_launches() - n0) // k

    with ClockSampler(0) as clk:
        ms_b, lb = timed(batched, a.steps)
    ms_p, lp = timed(plain, a.steps)
    de = sum(w * h * d for d in ds)
    print(json.dumps({"metric": "census capture MDE/s (Σ W·H·D_k per second), 10 pairs 2080x1560, batched", "value": de / (ms_b / 1e3) / 1e6,
                      "unit": "MDE/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_b, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "u8 cost / u16 aggregation", "data": "synthetic",
                      "config": {"workload": f"census capture: 10 pairs {w}x{h} on the reference grid, D {ds}, fused to one depth map",
                                 "launches_per_capture": {"batched": int(lb), "plain": int(lp)}},
                      "plain": {"ms_per_capture": ms_p, "mde_per_s": de / (ms_p / 1e3) / 1e6},
                      "gpu_launches": int(lb) * a.steps, "clocks": clk.summary()}))
    ctx.close()


def pyramid_job(a, w, h, steps, warmup, cpu=True):
    """DenseStereoPyramid.Run (DenseStereoSgm.cs:331-353) on a capture's reference group — five colour cameras of w x h
    (2080x1560: the finest layer is 2080x1560, as in StereoAsyncApi.State4And5) — then DenseUpsampleLayer.Run to 2w x 2h
    with a guide: the reference's whole dense job for one capture. Images on the device; ms per capture on the library's
    stream, per-layer device times and kernels; cpu: the oracle's pyramid on the host cores (cost prepass on every core,
    serial aggregation as the reference) on the same capture, as the job's CPU baseline."""
    import torch
    from lux_b200 import api, synth
    cap = synth.capture(w, h, 5, seed=3)
    torch.cuda.set_device(0)
    ctx = api.Context(0)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(lib.lux_sgm_stream(ctx.handle), device=torch.device("cuda", 0))
    d_imgs = [torch.from_numpy(im).cuda() for im in cap.images]
    guide = torch.from_numpy(np.random.default_rng(4).integers(0, 256, (2 * h, 2 * w, 4), dtype=np.uint8)).cuda()
    out = torch.empty((2 * h, 2 * w), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    info = []
    ups = []  # the upsample's (start, end) events of the timed steps

    def step(timed=False):
        layers = api.DenseStereoPyramid.run(d_imgs, cap.gray, cap.calibs, cap.near, cap.far, ctx=ctx)
        top = layers[-1]
        info[:] = [(L.W, L.H, L.n_planes, L.sgm_kernel, L.cost_kernel, L.gpu_ms_cost, L.gpu_ms_sgm, L.gpu_ms_wta, L.volume / (L.W * L.H))
                   for L in layers]
        gi = api.L.Img(guide.data_ptr(), 2 * w, 2 * h, 2 * w, 1)
        if timed:
            ups.append((torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)))
            ups[-1][0].record(stream)
        ctx.check(lib.lux_sgm_upsample(ctx.handle, top.device_ptr(0), top.W, top.H, 1, ctypes.byref(gi), w, h, 12.0, 2, None,
                                       out.data_ptr(), None))
        if timed:
            ups[-1][1].record(stream)
        for L in layers:
            L.close()

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    n0 = api.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        e0.record(stream)
        for _ in range(steps):
            step(timed=True)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    launches = api.kernel_launches() - n0
    ms_up = float(np.median([a.elapsed_time(b) for a, b in ups]))
    up_bytes = 2 * w * 2 * h * 8 + w * h * 8  # DenseUpsampleLayer: full-size depth out + guide in, layer depth in + shifted copy
    peak = float(peaks()["hbm_gbs"])
    ctx.close()
    de = sum(W * H * n for (W, H, n, *_) in info)
    res = {"workload": f"L16 pyramid on 5 colour cameras {w}x{h} + upsample to {2 * w}x{2 * h}", "ms_per_capture": ms,
           "captures_per_s": 1e3 / ms, "mde_per_s": de / (ms / 1e3) / 1e6, "gpu_launches": int(launches),
           "clocks": clk.summary(),
           "upsample": {"ms": ms_up, "gb_per_s": up_bytes / ms_up / 1e6, "frac": up_bytes / ms_up / 1e6 / peak,
                        "bytes": up_bytes, "note": "k_shift_resize + k_bilateral, of the measured HBM copy bandwidth"},
           "layers": [{"w": W, "h": H, "planes": n, "mean_cap": round(mc, 1), "sgm_kernel": sk, "cost_kernel": ck,
                       "ms_cost": round(c, 3), "ms_sgm": round(g, 3), "ms_wta": round(t, 3)}
                      for (W, H, n, sk, ck, c, g, t, mc) in info]}
    if cpu:
        from oracle import oracle as O
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        O.pyramid(cap.images, cap.gray, cap.calibs, cap.near, cap.far, threads=threads)
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": 1.0 / dt, "unit": "captures/s", "cores": threads, "kind": "port",
                               "sample": f"the same capture's DenseStereoPyramid.Run ({dt:.1f} s): oracle port, cost prepass on "
                                         f"{threads} threads, serial aggregation as the reference (the upsample not included)"}
    return res


def run_pyramid(a):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    w, h = (int(v) for v in a.pyramid_size.split("x"))
    r = pyramid_job(a, w, h, a.steps, a.warmup, cpu=not a.no_cpu_baseline)
    line = {"metric": f"capture dense jobs/s (DenseStereoPyramid.Run + upsample), 5 cameras {w}x{h}", "value": r["captures_per_s"],
            "unit": "captures/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": r["ms_per_capture"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8 cost / u16 aggregation",
            "data": "synthetic (colour capture, planar scene 0.4-6 m, 8-40 mm baselines)",
            "config": {"workload": r["workload"], "layers": r["layers"], "mde_per_s": r["mde_per_s"], "upsample": r["upsample"]},
            "gpu_launches": r["gpu_launches"], "clocks": r["clocks"]}
    if "cpu_baseline" in r:
        line["cpu_baseline"] = r["cpu_baseline"]
    print(json.dumps(line))


def main():
    a = args_()
    if a.pyramid:
        run_pyramid(a)
        return
    if a.census_capture:
        run_census_capture(a)
        return
    if a.census:
        run_census(a)
        return
    if a.stereo:
        run_stereo(a)
        return
    if a.cache:
        run_cache(a)
        return
    if a.sweep:
        run_sweep(a)
        return
    if a.serve:
        run_serve(a)
        return
    if a.impl == "reference":
        run_reference(a)
    else:
        run_lux(a)


if __name__ == "__main__":
    main()
