"""Benchmark of the B200 in-loop filter + film-grain path.

Metric: filtered Mpix/s (luma pixels of frames through the full configured
chain).  The headline workload is one 1920x1080 10-bit 4:2:0 frame per step
through deblock + CDEF + CCSO + loop restoration (NS/PC-Wiener, GDF), seeded
synthetic recon and side-info (no dataset is named; see rav2d_b200/synth.py).

  value       device-resident: recon and side-info staged in HBM before the
              timed region; each step filters a different resident frame
              (a ring larger than L2), timed with CUDA events.
  e2e         through the C ABI with pinned host buffers: every step uploads
              the recon and the side-info, filters and downloads the result.
  roofline    the dominant kernel's algorithmic bytes per launch over its
              event-timed average launch duration, against the measured HBM
              copy bandwidth.
  cpu_baseline  the CPU oracle (a restatement of the reference's scalar Rust
              filter path; the Rust reference cannot be built on this image)
              on a bounded sample of the same workload.

`--impl reference` times that CPU path alone with all host threads.
Multi-GPU: frames are independent, so N ranks run N replicas (no collective
on the data path); value = frames of all ranks / max rank time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W_, H_, BD_ = 1920, 1080, 10
SEED = 0x5EED0001
MPIX = W_ * H_ / 1e6
# algorithmic HBM bytes per luma pixel at 10-bit (4:2:0 = 1.5 samples / px,
# 2 B / sample): each stage reads its input frame once and writes its output
# once (3 + 3 B); loop restoration with chroma NS-Wiener and film grain also
# read the luma plane once more for the chroma planes' cross-component taps /
# scaling index (+2 B).  The deblock kernel runs both edge directions in one
# pass over the frame, so its minimum is one read and one write.
BYTES_PER_PX = {"deblock": 6.0, "cdef_ccso": 6.0, "loop_restoration": 8.0, "film_grain": 8.0}
# From one `ncu --set full` capture of each kernel on this workload (one
# launch each, `python -m rav2d_b200.profile --frames 24 --runs 2`): DRAM
# bytes read + written per launch (the outputs were still in L2 when the
# capture ended, so the write term was 0) and warp instructions per launch.
NCU_CAPTURE = {
    "commit": "b61cfe5 (deblock), 7a43533 (CDEF+CCSO), 2b0974d (LR)",
    "traffic": {"deblock": 6619904, "cdef_ccso": 6298624, "loop_restoration": 6847232},
    "warp_inst": {"deblock": 10063486, "cdef_ccso": 26085809, "loop_restoration": 26899014},
}
SMS = 148


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p:
            time.sleep(0.25)
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def make_inputs(n_distinct=4, db_blocks=False):
    """Seeded 1080p 10-bit frames; with db_blocks the deblock masks travel as
    the decoder's create_db_mask calls (a random partition of each frame)
    and are built on the device."""
    from rav2d_b200 import synth

    sfs = [synth.make_frame(W_, H_, BD_, SEED + 16 * i, chain="full") for i in range(n_distinct)]
    if db_blocks:
        for i, sf in enumerate(sfs):
            blocks, hdr = synth.make_db_blocks(np.random.default_rng(SEED + 16 * i + 1), W_, H_)
            sf.use_db_blocks(blocks, hdr)
    return sfs


def pinned_like(planes):
    import torch

    out = []
    for p in planes:
        t = torch.empty(p.shape, dtype=torch.int16 if p.dtype == np.uint16 else torch.uint8, pin_memory=True)
        a = t.numpy().view(p.dtype)
        a[:] = p
        out.append((t, a))
    return out


def run_ours(args, rank, world, device):
    import torch

    from rav2d_b200 import gpu

    torch.cuda.set_device(device)
    # a dedicated (non-default) stream: the library enqueues every kernel and
    # copy on it and the CUDA events below are recorded on it
    stream = torch.cuda.Stream(device)
    torch.cuda.set_stream(stream)
    ctx = gpu.Context(device)
    assert stream.cuda_stream != 0
    ctx.set_stream(stream.cuda_stream)
    sfs = make_inputs(db_blocks=True)
    # a ring of resident frames (larger than L2); the recon buffers are not
    # modified by filtering, so step i filters ring frame i % ring
    ring = args.ring
    frames = []
    for i in range(ring):
        fr = ctx.frame(W_, H_, BD_)
        sf = sfs[i % len(sfs)]
        fr.upload(sf.planes)
        fr.stage(sf)
        frames.append(fr)
    ctx.sync()
    torch.cuda.synchronize()

    from rav2d_b200 import replicas

    barrier = replicas.barrier

    # ---- device-resident timed region ----
    for i in range(args.warmup):
        frames[i % ring].run()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    l0 = ctx.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(device) as clk:
        time.sleep(1.0)  # let the sampler attach before the timed region
        ev0.record(stream)
        for i in range(args.steps):
            frames[i % ring].run()
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = ctx.launch_count() - l0
    ms = ev0.elapsed_time(ev1)
    barrier()
    units, ms_max, n_ranks = replicas.aggregate(MPIX * args.steps, ms, f"cuda:{device}")

    # ---- profiled pass: per-stage kernel durations from CUDA events ----
    ctx.profile(True)
    nprof = min(args.steps, 4 * ring)
    for i in range(nprof):
        frames[i % ring].run()
    prof = ctx.profile_read()
    ctx.profile(False)

    # ---- end to end through the ABI with pinned host buffers ----
    # every step uploads a frame's recon and side-info from pinned host
    # memory, filters it and downloads the result into pinned host memory.
    # With copy overlap (the default measurement) the uploads and downloads
    # run on the context's copy streams, so the transfers of one step overlap
    # the kernels of another; the serial variant keeps everything on one
    # stream.  The end event is recorded after a fence on every copy.
    pins = [pinned_like(sf.planes) for sf in sfs]
    # side-info records in page-locked memory too (a decoder would keep them
    # there): with copy overlap they are uploaded without staging
    import dataclasses

    def pinned_rec(a):
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        out = t.numpy().view(a.dtype).reshape(a.shape)
        out[...] = a
        return out

    def pinned_frame(sf, db):
        out = dataclasses.replace(sf, masks=pinned_rec(sf.masks), lr=pinned_rec(sf.lr), meta={})
        if db:
            out.use_db_blocks(pinned_rec(sf.meta["db_blocks"]), sf.meta["db_hdr"])
        return out

    sfs_db = [pinned_frame(sf, True) for sf in sfs]
    # the same frames with the edge masks built on the host (the masks cross
    # PCIe as given): the comparison the device mask build is for
    sfs_full = [pinned_frame(sf, False) for sf in sfs]
    sfs = sfs_db
    outs = [[a for _, a in pinned_like(sfs[0].planes)] for _ in range(4)]

    def e2e_step(i):
        k = i % len(sfs)
        fr = frames[i % ring]
        fr.upload([a for _, a in pins[k]])
        fr.stage(sfs[k])
        fr.run()
        fr.download_into(outs[i % len(outs)], 0)

    def e2e_run(n, overlap):
        ctx.overlap_copies(overlap)
        for i in range(args.warmup):
            e2e_step(i)
        ctx.sync()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(n):
            e2e_step(args.warmup + i)
        ctx.fence()
        e1.record(stream)
        torch.cuda.synchronize()
        ctx.sync()
        ms = e0.elapsed_time(e1)
        ctx.overlap_copies(False)
        u, ms_max, _ = replicas.aggregate(MPIX * n, ms, f"cuda:{device}")
        return u / (ms_max / 1e3)

    n_e2e = min(args.steps, 400)
    e2e_rate = e2e_run(n_e2e, True)
    e2e_serial_rate = e2e_run(min(n_e2e, 200), False)
    sfs = sfs_full
    e2e_full_rate = e2e_run(n_e2e, True)
    sfs = sfs_db
    recon_bytes = int(W_ * H_ * 1.5 * 2)
    # side-info crosses PCIe as the SB256 records without their edge masks
    # (12100 - 10240 bytes each), the restoration records packed to 960 bytes
    # per SB256 (the library packs them while staging) and the block records
    # (12 bytes per create_db_mask call, mean over the distinct frames)
    n_sb = sfs[0].masks.shape[0]
    rec_bytes = int(np.mean([sf.meta["db_blocks"].nbytes for sf in sfs]))
    side_bytes = int((12100 - 10240) * n_sb + 960 * n_sb + rec_bytes)
    side_bytes_full = int(sfs_full[0].masks.nbytes + 960 * n_sb)

    for fr in frames:
        fr.free()
    batch = run_batched(args, ctx, stream, device) if args.batch_steps > 0 else None
    uhd = run_4k_grain(args, ctx, stream, device) if args.grain_steps > 0 else None
    ctx.close()
    return {
        "batched": batch, "per_frame_4k_grain": uhd,
        "ms": ms_max, "units": units, "n_ranks": n_ranks, "launches": launches, "prof": prof, "nprof": nprof,
        "e2e_rate": e2e_rate, "n_e2e": n_e2e, "e2e_serial_rate": e2e_serial_rate,
        "e2e_full_rate": e2e_full_rate, "h2d_full": recon_bytes + side_bytes_full,
        "clocks": clk.summary(),
        "h2d": recon_bytes + side_bytes, "d2h": recon_bytes,
    }


MIX_RES = [(640, 360), (1280, 720), (1920, 1080), (3840, 2160)]


def make_mix(n=64, seed=0x5EED0003):
    """The batching workload: n frames, resolution drawn from MIX_RES, bit
    depth from {8, 10}, film grain on for a random half; full filter chain.
    Frames of the same (resolution, bit depth, grain) class share one seeded
    synthetic recon + side-info (the GPU does the same work either way)."""
    from rav2d_b200 import synth

    rng = np.random.default_rng(seed)
    specs = [(MIX_RES[rng.integers(len(MIX_RES))], int(rng.choice([8, 10])), bool(rng.integers(2))) for _ in range(n)]
    cache = {}
    out = []
    for wh, bd, g in specs:
        k = (wh, bd, g)
        if k not in cache:
            cache[k] = synth.make_frame(wh[0], wh[1], bd, seed + 0x100 + len(cache), chain="full", grain=g)
        out.append(cache[k])
    return out


def run_4k_grain(args, ctx, stream, device):
    """Per-frame 3840x2160 10-bit, full chain plus film grain (the reference's
    per-frame configuration with grain): a ring of 8 resident frames (1 GB,
    larger than L2), one frame filtered and grained per step."""
    import torch

    from rav2d_b200 import synth

    sfs = [synth.make_frame(3840, 2160, 10, 0x5EED0002 + 16 * i, chain="full", grain=True) for i in range(2)]
    ring = []
    for i in range(8):
        fr = ctx.frame(3840, 2160, 10)
        fr.upload(sfs[i % 2].planes)
        fr.stage(sfs[i % 2])
        ring.append(fr)
    ctx.sync()

    def step(i):
        sf = sfs[i % 8 % 2]
        ring[i % 8].run()
        ring[i % 8].grain(sf.fgd, sf.grain_seed)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    n = args.grain_steps
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(n):
        step(i)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / n
    for fr in ring:
        fr.free()
    return {"workload": "per-frame 3840x2160 10-bit, deblock+CDEF+CCSO+LR+film grain, resident ring of 8 frames",
            "steps": n, "ms_per_frame": round(ms, 4), "value": round(3840 * 2160 / 1e6 / ms * 1e3, 1),
            "unit": "Mpix/s"}


def run_batched(args, ctx, stream, device):
    """64-frame mixed workload: one batch (one persistent launch per stage,
    CUDA graph) per step vs the per-frame pipeline over the same frames."""
    import torch

    sfs = make_mix()
    frames = []
    for sf in sfs:
        fr = ctx.frame(sf.width, sf.height, sf.bitdepth)
        fr.upload(sf.planes)
        fr.stage(sf)
        frames.append(fr)
    ctx.sync()
    mpix = sum(sf.width * sf.height for sf in sfs) / 1e6
    items = list(zip(frames, sfs))

    def per_frame():
        for fr, sf in items:
            fr.run()
            if sf.fgd is not None:
                fr.grain(sf.fgd, sf.grain_seed)

    def batched():
        ctx.batch_submit(items, staged=True)

    def timed(fn, reps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        l0 = ctx.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, (ctx.launch_count() - l0) / reps

    reps = max(3, min(args.batch_steps, args.steps))
    pf_ms, pf_l = timed(per_frame, reps)
    b_ms, b_l = timed(batched, reps)
    sms, cfg = ctx.batch_config()
    tile_rows = ctx.batch_tile_rows()
    for fr in frames:
        fr.free()
    by_class = run_batched_by_class(args, ctx, timed, reps)
    mix = {}
    for sf in sfs:
        k = f"{sf.width}x{sf.height}/{sf.bitdepth}bit{'+grain' if sf.fgd is not None else ''}"
        mix[k] = mix.get(k, 0) + 1
    return {
        "workload": "64 frames/batch, resolutions {640x360,1280x720,1920x1080,3840x2160} x {8,10}-bit, "
                    "full chain, film grain on a random half", "mix": mix,
        "mpix_per_batch": round(mpix, 3), "steps": reps,
        "value": round(mpix / b_ms * 1e3, 2), "unit": "Mpix/s", "ms_per_batch": round(b_ms, 4),
        "launches_per_batch": b_l,
        "per_frame_value": round(mpix / pf_ms * 1e3, 2), "per_frame_ms": round(pf_ms, 4),
        "per_frame_launches": pf_l,
        "speedup_vs_per_frame": round(pf_ms / b_ms, 3), "ctas_per_sm": cfg, "tile_rows": tile_rows, "sms": sms,
        "l2": f"inputs larger than L2: {round(mpix * 1.5 * 1.5, 0)} MB of recon per batch",
        "by_class": by_class,
    }


# frames per batch of each (resolution, bit depth) class: about 15 Mpix each
CLASS_FRAMES = {(640, 360): 64, (1280, 720): 16, (1920, 1080): 8, (3840, 2160): 2}


def run_batched_by_class(args, ctx, timed, reps):
    """Batched vs per-frame for one resolution and bit depth at a time (full
    filter chain, no grain): where batching can win is the small frames,
    whose per-frame grids fill a fraction of the GPU."""
    from rav2d_b200 import synth

    out = {}
    for (w, h), n in CLASS_FRAMES.items():
        for bd in (8, 10):
            sf = synth.make_frame(w, h, bd, 0x5EED3000 + w + bd, chain="full")
            frames = []
            for _ in range(n):
                fr = ctx.frame(w, h, bd)
                fr.upload(sf.planes)
                fr.stage(sf)
                frames.append(fr)
            ctx.sync()
            items = [(fr, sf) for fr in frames]

            def per_frame():
                for fr in frames:
                    fr.run()

            def batched():
                ctx.batch_submit(items, staged=True)

            pf_ms, _ = timed(per_frame, reps)
            b_ms, _ = timed(batched, reps)
            for fr in frames:
                fr.free()
            mpix = n * w * h / 1e6
            out[f"{w}x{h}/{bd}bit"] = {"frames": n, "per_frame_mpix_s": round(mpix / pf_ms * 1e3, 1),
                                       "batched_mpix_s": round(mpix / b_ms * 1e3, 1),
                                       "speedup": round(pf_ms / b_ms, 3)}
    return out


def run_serving(args, device):
    """32 streams, resolutions 360p..4K, 8/10-bit, film grain on half the
    streams; each stream's frames arrive as a Poisson process at 30 fps and
    go through the continuous-batching server (40 GB device budget, pinned
    host buffers).  A warm-up second fills the streams' resident frames and
    the autotuner cache, then the statistics are reset and the measured
    window runs for --serve-seconds."""
    import heapq

    import torch

    from rav2d_b200 import gpu, synth

    rng = np.random.default_rng(0x5EED0004)
    n_streams, fps = 32, 30.0
    specs = [(MIX_RES[k % len(MIX_RES)], 8 + 2 * ((k // len(MIX_RES)) % 2), k % 2 == 0) for k in range(n_streams)]
    cache = {}
    for wh, bd, g in specs:
        if (wh, bd, g) not in cache:
            sf = synth.make_frame(wh[0], wh[1], bd, 0x5EED2000 + len(cache), chain="full", grain=g)
            cache[(wh, bd, g)] = (sf, [a for _, a in pinned_like(sf.planes)])
    outs = [[[a for _, a in pinned_like(cache[sp][0].planes)] for _ in range(4)] for sp in specs]
    ctx = gpu.Context(device)
    srv = gpu.Server(ctx, mem_budget=40 << 30, max_batch=64)
    results = []
    lock = threading.Lock()

    def drive(seconds):
        heap = [(rng.exponential(1.0 / fps), k) for k in range(n_streams)]
        heapq.heapify(heap)
        t0 = time.perf_counter()
        ids = []
        cnt = [0] * n_streams
        while True:
            t, k = heapq.heappop(heap)
            if t > seconds:
                break
            dt = t0 + t - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            sf, src = cache[specs[k]]
            ids.append(srv.submit(k, sf, src, outs[k][cnt[k] % 4]))
            cnt[k] += 1
            heapq.heappush(heap, (t + rng.exponential(1.0 / fps), k))
        return ids

    def collect(ids):
        for rid in ids:
            rc, res = srv.wait(rid, 60000)
            with lock:
                results.append((rc, res.status, res.latency_us, res.batch_frames))

    collect(drive(1.0))
    srv.stats(reset=True)
    results.clear()
    with ClockSampler(device) as clk:
        ids = drive(args.serve_seconds)
        collect(ids)
    st = srv.stats()
    srv.close()
    ctx.close()
    torch.cuda.synchronize()
    offered = sum(w * h for (w, h), _, _ in specs) * fps / 1e6
    ok = [r for r in results if r[0] == 0 and r[1] == 0]
    return {
        "workload": "32 streams x 30 fps Poisson arrivals, 360p/720p/1080p/4K x 8/10-bit, full chain, film grain "
                    "on half the streams, 40 GB device budget, continuous batching (<=64 frames/batch)",
        "seconds": args.serve_seconds, "frames": len(results), "ok": len(ok),
        "offered_mpix_s": round(offered, 1),
        "value": round(st["mpix"] / st["span_s"], 1) if st["span_s"] else None, "unit": "Mpix/s",
        "p50_ms": round(st["p50_us"] / 1e3, 3), "p99_ms": round(st["p99_us"] / 1e3, 3),
        "mean_ms": round(st["mean_us"] / 1e3, 3), "max_ms": round(st["max_us"] / 1e3, 3),
        "batches": st["batches"], "mean_batch": round(st["mean_batch"], 2),
        "resident_gb": round(st["resident_bytes"] / 2 ** 30, 2), "evictions": st["evictions"],
        "latency": "submit -> display frame in pinned host memory (upload, filter, grain, download)",
        "clocks": clk.summary(),
    }


def cpu_baseline(seconds=12.0, threads=1):
    """The oracle on `threads` host threads, one frame per thread, for about
    `seconds`; returns (Mpix/s, frames, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    sfs = make_inputs(2)
    pyoracle.lib()
    done = [0]
    lock = threading.Lock()
    t0 = time.time()

    def worker(k):
        while time.time() - t0 < seconds:
            pyoracle.filter_frame(sfs[k % len(sfs)])
            with lock:
                done[0] += 1

    ths = [threading.Thread(target=worker, args=(k,)) for k in range(threads)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    dt = time.time() - t0
    return done[0] * MPIX / dt, done[0], dt


def reference_arm(args, config, metric):
    """The reference's CPU filter path (the oracle: the Rust reference cannot
    be built here) on all host threads, on the same workload.  Each step
    filters one sample frame per thread: 1920 x `rows` 10-bit with the full
    chain, `rows` chosen so the whole --steps/--warmup run takes about
    --ref-seconds (whole 1080p frames when the step count allows)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from concurrent.futures import ThreadPoolExecutor

    from rav2d_b200 import synth

    pyoracle.lib()
    nthreads = os.cpu_count() or 1
    full = make_inputs(1)[0]
    t = time.perf_counter()
    pyoracle.filter_frame(full)
    rate = MPIX / (time.perf_counter() - t)  # Mpix/s on one thread
    per_step = args.ref_seconds * rate / (args.steps + args.warmup)
    rows = int(min(H_, max(64, per_step * 1e6 / W_))) // 8 * 8
    samples = [synth.make_frame(W_, rows, BD_, SEED + 16 * k, chain="full") for k in range(min(nthreads, 4))]
    mpix_step = nthreads * W_ * rows / 1e6
    times = []
    with ThreadPoolExecutor(nthreads) as pool:
        for i in range(args.warmup + args.steps):
            t = time.perf_counter()
            list(pool.map(lambda k: pyoracle.filter_frame(samples[k % len(samples)]), range(nthreads)))
            if i >= args.warmup:
                times.append(time.perf_counter() - t)
    tot = sum(times)
    val = mpix_step * len(times) / tot
    sample = (f"each step: one 1920x{rows} 10-bit frame (full chain) per host thread through the oracle (C++ "
              f"restatement of the reference scalar Rust filter path), {nthreads} threads")
    return {"impl": "reference", "metric": metric, "value": round(val, 3), "unit": "Mpix/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1000 * tot / len(times), 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u16", "data": "synthetic", "config": config,
            "cpu_baseline": {"value": round(val, 3), "unit": "Mpix/s", "cores": nthreads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(val, 3), "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--ring", type=int, default=48)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--batch-steps", type=int, default=30, help="timed batches of the 64-frame mix (0 = skip)")
    ap.add_argument("--grain-steps", type=int, default=300,
                    help="timed frames of the per-frame 4K 10-bit + film grain block (0 = skip)")
    ap.add_argument("--serve-seconds", type=float, default=5.0, help="measured serving window (0 = skip)")
    ap.add_argument("--ref-seconds", type=float, default=120.0, help="target duration of --impl reference")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    from rav2d_b200 import replicas

    replicas.check_world(args.gpus)
    rank, world, local = replicas.env()
    config = {"workload": "per-frame 1920x1080 10-bit 4:2:0, deblock+CDEF+CCSO+LR(NS/PC-Wiener+GDF), no grain",
              "frames_per_step": 1, "width": W_, "height": H_, "bitdepth": BD_, "inloop_mask": 31,
              "l2": "inputs larger than L2: a ring of 48 resident frames (~330 MB), step i filters frame i % 48",
              "parallelism": f"replicas{args.gpus}"}
    metric = "filtered Mpix/s (luma), 10-bit per-frame pipeline on 1 B200"

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(reference_arm(args, config, metric)), flush=True)
        return

    import torch

    replicas.init("nccl")
    res = run_ours(args, rank, world, local)
    res["serving"] = run_serving(args, local) if args.serve_seconds > 0 and rank == 0 else None
    replicas.finish()
    if rank != 0:
        return
    n = res["n_ranks"]
    ms_step = res["ms"] / args.steps
    value = res["units"] / (res["ms"] / 1e3)
    e2e = res["e2e_rate"]
    prof = res["prof"]
    dom = max((k for k in prof if prof[k][1] > 0), key=lambda k: prof[k][0])
    dom_ms, dom_n = prof[dom]
    avg_launch_s = dom_ms / dom_n / 1e3
    achieved = BYTES_PER_PX[dom] * W_ * H_ / avg_launch_s / 1e9
    stages_us = {k: round(v[0] / max(1, res["nprof"]) * 1e3, 2) for k, v in prof.items() if v[1]}
    sm_mhz = (res["clocks"] or {}).get("sm_mhz")
    peak, peak_kind = peaks()
    cpu_v, cpu_n, cpu_dt = cpu_baseline(seconds=args.cpu_seconds, threads=1)
    ncores = os.cpu_count() or 1
    cpu_all = cpu_baseline(seconds=min(args.cpu_seconds, 6.0), threads=ncores) if args.cpu_seconds >= 1 else None
    line = {
        "metric": metric, "value": round(value, 2), "unit": "Mpix/s", "n_gpus": n, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 5), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16", "data": "synthetic (seeded recon + side-info, rav2d_b200/synth.py)",
        "config": config,
        "e2e": {"value": round(e2e, 2), "unit": "Mpix/s", "h2d_bytes_per_step": res["h2d"],
                "d2h_bytes_per_step": res["d2h"], "steps": res["n_e2e"],
                "path": "r2g_frame_upload_recon + r2g_frame_stage + r2g_frame_run + r2g_download, pinned host, "
                        "copies overlapped with kernels (r2g_ctx_overlap_copies); deblock edge masks built on "
                        "the device from the decoder's create_db_mask calls (R2gSideInfo.db_masks)",
                "serial_value": round(res["e2e_serial_rate"], 2),
                "host_masks": {"value": round(res["e2e_full_rate"], 2), "h2d_bytes_per_step": res["h2d_full"],
                               "path": "the same, with the edge masks built on the host and uploaded"}},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "traffic": NCU_CAPTURE["traffic"].get(dom),
                     "traffic_source": "ncu dram__bytes_read.sum+dram__bytes_write.sum, one launch, from a capture "
                                       "of commit " + NCU_CAPTURE["commit"],
                     "bytes_per_launch": int(BYTES_PER_PX[dom] * W_ * H_),
                     "avg_launch_us": round(avg_launch_s * 1e6, 2)},
        "stages_us_per_frame": stages_us,
        # the bound that limits these stages: integer issue, warp
        # instructions / (SMs x 4 schedulers x median SM clock x stage time)
        "issue_roofline": {
            k: {"warp_inst": NCU_CAPTURE["warp_inst"][k], "stage_us": stages_us[k],
                "frac": round(NCU_CAPTURE["warp_inst"][k] / (SMS * 4 * sm_mhz * 1e6 * stages_us[k] * 1e-6), 3)}
            for k in NCU_CAPTURE["warp_inst"] if k in stages_us and sm_mhz},
        "issue_roofline_source": "warp instructions per launch from a one-kernel ncu capture of commit "
                                 + NCU_CAPTURE["commit"] + "; stage times and SM clock from this run",
        "cpu_baseline": {"value": round(cpu_v, 3), "unit": "Mpix/s", "cores": 1, "kind": "port",
                         "sample": f"{cpu_n} whole 1080p 10-bit frames through the oracle (C++ restatement of the "
                                   f"reference scalar Rust filter path) on 1 host core in {cpu_dt:.1f} s"},
        "cpu_all_cores": ({"value": round(cpu_all[0], 3), "unit": "Mpix/s", "cores": ncores, "kind": "port",
                           "sample": f"{cpu_all[1]} whole 1080p frames, one per thread, in {cpu_all[2]:.1f} s"}
                          if cpu_all else None),
        "clocks": res["clocks"], "gpu_launches": res["launches"],
        "batched": res["batched"], "per_frame_4k_grain": res["per_frame_4k_grain"], "serving": res["serving"],
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
