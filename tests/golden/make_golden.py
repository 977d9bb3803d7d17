"""Writes tests/golden/oracle_digests.json: SHA-256 digests of the oracle's
output planes (filtered and, where film grain is on, grained) on seeded
synthetic frames.  The oracle is the C++ restatement of the reference's
scalar filter path (oracle/); the reference itself (Rust) cannot run here.

The GPU tests compare the CUDA path against these committed digests, and
the CPU tests re-derive them from the oracle, so a change to either the
oracle or the synthetic generator shows up as a digest mismatch.

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

# (name, width, height, bitdepth, chain, grain, seed)
CASES = [
    ("db_64x64_8", 64, 64, 8, "db", False, 0x601D0001),
    ("plain_352x288_8", 352, 288, 8, "db_cdef", False, 0x5EED0000),
    ("full_72x40_8", 72, 40, 8, "full", False, 0x601D0003),
    ("full_128x128_10", 128, 128, 10, "full", False, 0x601D0004),
    ("full_grain_160x96_10", 160, 96, 10, "full", True, 0x601D0005),
    ("full_grain_200x120_8", 200, 120, 8, "full", True, 0x601D0006),
]


def frame(case):
    from rav2d_b200 import synth

    _, w, h, bd, chain, grain, seed = case
    return synth.make_frame(w, h, bd, seed, chain=chain, grain=grain)


def digest(planes, sf):
    out = []
    for pl, p in enumerate(planes):
        hh, ww = sf.height >> (pl > 0), sf.width >> (pl > 0)
        out.append(hashlib.sha256(p[:hh, :ww].astype("<u2").tobytes()).hexdigest())
    return out


def oracle_digests(case):
    import pyoracle

    sf = frame(case)
    f = pyoracle.filter_frame(sf)
    d = {"filtered": digest(f, sf)}
    if sf.fgd is not None:
        d["grained"] = digest(pyoracle.apply_grain(sf, f), sf)
    return d


def main():
    out = {c[0]: dict(oracle_digests(c), spec=list(c[1:])) for c in CASES}
    with open(os.path.join(HERE, "oracle_digests.json"), "w") as fp:
        json.dump(out, fp, indent=1, sort_keys=True)
        fp.write("\n")


if __name__ == "__main__":
    main()
