"""Run one fixed workload of the filter path, for an external profiler.

    python -m rav2d_b200.profile --width 1920 --height 1080 --bitdepth 10 \
        --frames 24 --runs 2 [--db-blocks] [--grain]

Allocates a ring of `frames` device-resident frames (seeded synthetic recon
and side-info, as the bench uses), stages each once (with --db-blocks the
deblock masks are built on the device from block records), then runs every
frame of the ring `runs` times in order and synchronises.  The kernel launch
order per frame is deblock, CDEF+CCSO, loop restoration (then film grain
with --grain), so a profiler's launch index selects a stage of a given
frame: the last ring pass reads frames that are no longer in L2 once the
ring is larger than 126 MB.  Prints one line: the launches and the wall
time (not a measurement: use CUDA events or the bench for timings).
"""
import argparse
import time

import numpy as np

from . import gpu, synth


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--bitdepth", type=int, default=10)
    ap.add_argument("--frames", type=int, default=24)
    ap.add_argument("--runs", type=int, default=2)
    ap.add_argument("--seed", type=int, default=0x5EED0001)
    ap.add_argument("--db-blocks", action="store_true")
    ap.add_argument("--grain", action="store_true")
    args = ap.parse_args()
    ctx = gpu.Context(0)
    sfs = [synth.make_frame(args.width, args.height, args.bitdepth, args.seed + i, grain=args.grain)
           for i in range(min(args.frames, 4))]
    if args.db_blocks:
        for i, sf in enumerate(sfs):
            blocks, hdr = synth.make_db_blocks(np.random.default_rng(args.seed + 100 + i), args.width, args.height)
            sf.use_db_blocks(blocks, hdr)
    frames = []
    for i in range(args.frames):
        sf = sfs[i % len(sfs)]
        fr = ctx.frame(args.width, args.height, args.bitdepth)
        fr.upload(sf.planes)
        fr.stage(sf)
        frames.append((fr, sf))
    ctx.sync()
    l0 = ctx.launch_count()
    t0 = time.perf_counter()
    for _ in range(args.runs):
        for fr, sf in frames:
            fr.run()
            if args.grain:
                fr.grain(sf.fgd, sf.grain_seed)
    ctx.sync()
    dt = time.perf_counter() - t0
    print(f"profile: {args.runs} x {args.frames} frames {args.width}x{args.height} {args.bitdepth}-bit, "
          f"{ctx.launch_count() - l0} launches, {dt * 1e3:.1f} ms wall", flush=True)
    for fr, _ in frames:
        fr.free()
    ctx.close()


if __name__ == "__main__":
    main()
