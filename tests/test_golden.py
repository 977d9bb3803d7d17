"""Committed golden digests (tests/golden/oracle_digests.json, written by
tests/golden/make_golden.py from the oracle on seeded synthetic frames).

CPU: the oracle re-derives every digest (guards the oracle and the
generator against silent drift).  GPU: the CUDA path's output planes hash
to the same digests (tolerance 0: integer path)."""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden  # noqa: E402

with open(os.path.join(HERE, "golden", "oracle_digests.json")) as fp:
    GOLDEN = json.load(fp)

CASES = {c[0]: c for c in make_golden.CASES}


def test_cases_and_fixture_agree():
    assert sorted(GOLDEN) == sorted(CASES)
    for name, c in CASES.items():
        assert GOLDEN[name]["spec"] == list(c[1:])


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_golden(oracle, name):
    d = make_golden.oracle_digests(CASES[name])
    assert d["filtered"] == GOLDEN[name]["filtered"]
    assert d.get("grained") == GOLDEN[name].get("grained")


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_matches_golden(name):
    from rav2d_b200 import gpu

    sf = make_golden.frame(CASES[name])
    ctx = gpu.Context(0)
    try:
        if sf.fgd is not None:
            f, g = gpu.filter_frame(ctx, sf, grain=True)
            assert make_golden.digest(g, sf) == GOLDEN[name]["grained"]
        else:
            f = gpu.filter_frame(ctx, sf)
        assert make_golden.digest(f, sf) == GOLDEN[name]["filtered"]
    finally:
        ctx.close()
