"""The reference's unit tests of the dequantiser lookup the deblocking
thresholds use (crates/rav2d/src/quantizer.rs tests test_dq_lookup_*) and of
the GDF table sizes (crates/rav2d/src/gdf_tables.rs tests), re-asserted
against the oracle's dq_lookup (oracle/deblock.cpp) and the generated table
header both the oracle and the CUDA kernels compile (rav2d_b200/csrc/
av2_tables.h).  The quantizer file's quantisation-matrix tests (untriangle,
transpose, subsample, init_qm_tables, qm_tbl_*) cover dequantisation, which
is not on the filter path."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _sizes():
    hdr = open(os.path.join(ROOT, "rav2d_b200", "csrc", "av2_tables.h")).read()
    return {m.group(1): int(m.group(2)) for m in re.finditer(r"X\((\w+), (\d+), 0x[0-9a-f]+ULL\)", hdr)}


def test_dq_lookup_zero(oracle):
    """quantizer.rs:1893-1896"""
    assert oracle.lib().r2o_dq_lookup(0) == 64


def test_dq_lookup_first_entries(oracle):
    """quantizer.rs:1898-1908"""
    L = oracle.lib()
    assert [L.r2o_dq_lookup(q) for q in (1, 2, 12, 24)] == [40, 41, 55, 78]


def test_dq_lookup_second_shift(oracle):
    """quantizer.rs:1910-1916"""
    L = oracle.lib()
    assert L.r2o_dq_lookup(25) == 80 and L.r2o_dq_lookup(26) == 82


def test_dq_lookup_higher_shifts(oracle):
    """quantizer.rs:1918-1922"""
    assert oracle.lib().r2o_dq_lookup(49) == 160


def test_gdf_alpha_size():
    """gdf_tables.rs:2639-2642"""
    assert _sizes()["GDF_ALPHA"] == 3168


def test_gdf_weight_size():
    """gdf_tables.rs:2644-2647"""
    assert _sizes()["GDF_WEIGHT"] == 9504


def test_gdf_intra_error_size():
    """gdf_tables.rs:2649-2652"""
    assert _sizes()["GDF_INTRA_ERROR"] == 24576


def test_gdf_inter_error_size():
    """gdf_tables.rs:2654-2657"""
    assert _sizes()["GDF_INTER_ERROR"] == 30000
