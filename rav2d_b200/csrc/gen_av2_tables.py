#!/usr/bin/env python3
"""Extract the AV2 in-loop-filter constant tables from the rav2d Rust sources
into a C header shared by the CUDA kernels and the CPU oracle.

The tables are normative AV2 data (deblock side thresholds, CCSO quantiser and
offset tables, PC-Wiener filter banks and classifiers, GDF alpha/weight/bias/
error tables, the film-grain Gaussian sequence).  They must be bit-identical
to the reference, so they are read from its sources rather than retyped:

  crates/rav2d/src/tables.rs      (BSD-2-Clause, rav2d contributors)
  crates/rav2d/src/gdf_tables.rs  (BSD-2-Clause, rav2d contributors)

Usage:  python gen_av2_tables.py <rav2d checkout> <output header>

The output header is committed; this script only needs to be re-run when the
reference tables change.  Each table is checked against the element count
declared in its Rust type, and a FNV-1a digest of every table is written into
the header so tests can detect a stale or hand-edited copy.
"""
import re
import sys
from pathlib import Path

# (rust file, rust name, C element type)
TABLES = [
    ("tables.rs", "CDEF_DIRECTIONS", "int8_t"),
    ("tables.rs", "CCSO_QUANT_SZ", "uint16_t"),
    ("tables.rs", "CCSO_OFFSET", "int8_t"),
    ("tables.rs", "NS_WIENER_COEF_RANGE_Y", "int8_t"),
    ("tables.rs", "NS_WIENER_COEF_RANGE_UV", "int8_t"),
    ("tables.rs", "DEBLOCK_SIDE_THRESHOLDS", "int16_t"),
    ("tables.rs", "WIENER_NS_FILTERS", "int8_t"),
    ("tables.rs", "PC_WIENER_FILTERS", "int16_t"),
    ("tables.rs", "PC_WIENER_SUB_CLASSIFY", "uint8_t"),
    ("tables.rs", "PC_WIENER_SUB_CLASSIFY_NS", "uint8_t"),
    ("tables.rs", "GAUSSIAN_SEQUENCE", "int16_t"),
    ("tables.rs", "PC_WIENER_LUT_TO_CLASS", "uint8_t"),
    ("gdf_tables.rs", "GDF_ALPHA", "uint16_t"),
    ("gdf_tables.rs", "GDF_WEIGHT", "int16_t"),
    ("gdf_tables.rs", "GDF_BIAS", "int16_t"),
    ("gdf_tables.rs", "GDF_INTRA_ERROR", "int8_t"),
    ("gdf_tables.rs", "GDF_INTER_ERROR", "int8_t"),
    # block / transform geometry read by the deblock mask builder
    # (lf_mask.rs create_db_mask, mask_edges_part)
    ("tables.rs", "BLOCK_DIMENSIONS", "uint8_t"),
    ("tables.rs", "TXFM_DIMENSIONS", "uint8_t"),
    ("tables.rs", "MAX_TXFM_SIZE_FOR_BS", "uint8_t"),
    ("tables.rs", "TX_PART_TBL", "int8_t"),
]

# Named array lengths and struct element sizes used in the tables' Rust types
# (levels.rs N_BS_SIZES / N_RECT_TX_SIZES; tables.rs TxfmInfo has 8 u8 fields).
CONSTS = {"N_BS_SIZES": 31, "N_RECT_TX_SIZES": 25}
STRUCT_FIELDS = {"TxfmInfo": 8}


def parse_table(src: str, name: str):
    m = re.search(r"pub\s+(?:static|const)\s+" + name + r"\s*:\s*(.+?)\s*=\s*\[", src)
    if not m:
        raise SystemExit(f"table {name} not found")
    rust_type = m.group(1)
    start = m.end() - 1
    depth = 0
    end = None
    for i in range(start, len(src)):
        c = src[i]
        if c == "[":
            depth += 1
        elif c == "]":
            depth -= 1
            if depth == 0:
                end = i + 1
                break
    body = src[start:end]
    body = re.sub(r"//[^\n]*", "", body)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    vals = [int(v) for v in re.findall(r"-?\d+", body)]
    dims = []
    t = rust_type.strip()
    while t.startswith("["):
        inner, _, n = t[1:-1].rpartition(";")
        n = n.strip()
        dims.append(CONSTS[n] if n in CONSTS else int(n))
        t = inner.strip()
    if t in STRUCT_FIELDS:
        dims.append(STRUCT_FIELDS[t])
    count = 1
    for d in dims:
        count *= d
    if len(vals) != count:
        raise SystemExit(f"{name}: {len(vals)} values, type {rust_type} wants {count}")
    return dims, vals


def fnv1a(vals):
    h = 0xCBF29CE484222325
    for v in vals:
        for b in (v & 0xFFFFFFFF).to_bytes(4, "little"):
            h ^= b
            h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


def main():
    root = Path(sys.argv[1]) / "crates" / "rav2d" / "src"
    out = Path(sys.argv[2])
    srcs = {}
    lines = [
        "/* Generated by gen_av2_tables.py from the rav2d sources",
        " * (crates/rav2d/src/tables.rs, crates/rav2d/src/gdf_tables.rs).",
        " * Copyright (c) 2026, rav2d contributors. BSD-2-Clause:",
        " * redistributions of source code must retain this notice.",
        " *",
        " * Include after defining R2G_TABLE(type, name) to pick the storage",
        " * qualifier and the symbol name (host: static const; device: __device__).",
        " * Do not edit by hand. */",
        "#include <stdint.h>",
        "",
    ]
    digests = []
    for fname, name, ctype in TABLES:
        if fname not in srcs:
            srcs[fname] = (root / fname).read_text()
        dims, vals = parse_table(srcs[fname], name)
        decl = "".join(f"[{d}]" for d in dims)
        lines.append(f"R2G_TABLE({ctype}, {name}){decl} = {{")
        # flat brace-initialisation is valid C/C++ for multi-dim arrays
        for i in range(0, len(vals), 20):
            lines.append("    " + ", ".join(str(v) for v in vals[i:i + 20]) + ",")
        lines.append("};")
        lines.append("")
        digests.append((name, len(vals), fnv1a(vals)))
    lines.append("#ifndef R2G_TABLE_DIGESTS_DEFINED")
    lines.append("#define R2G_TABLE_DIGESTS_DEFINED")
    lines.append("/* name, element count, FNV-1a 64 over little-endian int32 values */")
    lines.append("#define R2G_TABLE_DIGEST_LIST \\")
    for name, n, h in digests:
        lines.append(f"    X({name}, {n}, 0x{h:016x}ULL) \\")
    lines.append("")
    lines.append("#endif")
    out.write_text("\n".join(lines) + "\n")
    print(f"wrote {out}: {len(TABLES)} tables")


if __name__ == "__main__":
    main()
