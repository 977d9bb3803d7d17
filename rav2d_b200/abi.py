"""ctypes / numpy mirrors of the C ABI in include/rav2d_gpu.h.

The per-SB256 side-info records are numpy structured dtypes (so whole frames
of masks are one contiguous array); the frame-constant parameter blocks are
ctypes structures.  Both reproduce the C layout byte for byte; `check_sizes`
compares them against the library's own `sizeof` values.
"""
import ctypes as C

import numpy as np

R2G_OK = 0
R2G_E_INVALID = -1
R2G_E_OOM = -2
R2G_E_TIMEOUT = -3
R2G_E_DEVICE = -4
R2G_E_NOTREADY = -5
R2G_E_TOO_LARGE = -6

INLOOP_DEBLOCK = 1 << 0
INLOOP_CDEF = 1 << 1
INLOOP_CCSO = 1 << 2
INLOOP_WIENER = 1 << 3
INLOOP_GDF = 1 << 4
INLOOP_ALL = 0x1F

RESTORE_NONE = 0
RESTORE_PC_WIENER = 1
RESTORE_NS_WIENER = 2
RESTORE_SWITCHABLE = 3

# R2gAv2Filter (mirrors Av2Filter, lf_mask.rs:8-19)
AV2_FILTER_DTYPE = np.dtype([
    ("filter_y", "<u2", (2, 64, 5, 4)),
    ("filter_uv", "<u2", (2, 64, 5, 4)),
    ("qidx", "<u2", (16,)),
    ("gdf", "u1", (16,)),
    ("cdef_idx", "i1", (16,)),
    ("ccso", "u1", (3,)),
    ("_pad0", "u1"),
    ("noskip_mask", "<u2", (32, 4)),
    ("lr_noskip_mask", "<u2", (64, 4)),
    ("lossless_mask_y", "<u2", (64, 4)),
    ("lossless_mask_uv", "<u2", (64, 4)),
])
assert AV2_FILTER_DTYPE.itemsize == 12100

# R2gAv2RestorationUnit / R2gAv2Restoration (lf_mask.rs:2-5, :39-41)
LR_UNIT_DTYPE = np.dtype([("restoration_type", "u1"), ("ns_filter", "i1", (16, 32))])
assert LR_UNIT_DTYPE.itemsize == 513
AV2_RESTORATION_DTYPE = np.dtype([("lr", LR_UNIT_DTYPE, (3, 16))])
assert AV2_RESTORATION_DTYPE.itemsize == 513 * 48


class CcsoPlane(C.Structure):
    _fields_ = [
        ("enabled", C.c_uint8),
        ("bo_only", C.c_uint8),
        ("scale_idx", C.c_uint8),
        ("quant_idx", C.c_uint8),
        ("ext_filter_support", C.c_uint8),
        ("edge_clf", C.c_uint8),
        ("max_band_log2", C.c_uint8),
        ("_pad0", C.c_uint8),
        ("filter_off", C.c_uint8 * 64),
    ]


class RestorationPlane(C.Structure):
    _fields_ = [
        ("restoration_type", C.c_uint8),
        ("frame_filters_on", C.c_uint8),
        ("num_classes_idx", C.c_uint8),
        ("num_classes", C.c_uint8),
        ("filter", (C.c_int8 * 18) * 16),
    ]


class FrameParams(C.Structure):
    _fields_ = [
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("bitdepth", C.c_int32),
        ("layout", C.c_int32),
        ("sb128", C.c_int32),
        ("cfl_ds_filter_index", C.c_int32),
        ("deblock_level_y", C.c_uint8 * 2),
        ("deblock_level_u", C.c_uint8),
        ("deblock_level_v", C.c_uint8),
        ("deblock_delta_q_y", C.c_int8 * 2),
        ("deblock_delta_q_u", C.c_int8),
        ("deblock_delta_q_v", C.c_int8),
        ("quant_yac", C.c_int32),
        ("quant_uac_delta", C.c_int8),
        ("quant_vac_delta", C.c_int8),
        ("seg_enabled", C.c_uint8),
        ("_pad0", C.c_uint8),
        ("seg_delta_q", C.c_int16 * 8),
        ("seg_lossless", C.c_uint8 * 8),
        ("seq_cdef", C.c_uint8),
        ("cdef_damping", C.c_uint8),
        ("cdef_on_skiptx", C.c_uint8),
        ("cdef_n_strengths", C.c_uint8),
        ("cdef_y_strength", C.c_uint8 * 8),
        ("cdef_uv_strength", C.c_uint8 * 8),
        ("ccso", CcsoPlane * 3),
        ("restoration", RestorationPlane * 3),
        ("restoration_unit_size", C.c_uint8 * 2),
        ("gdf_enabled", C.c_uint8),
        ("gdf_qp_idx", C.c_uint8),
        ("gdf_scale", C.c_uint8),
        ("frame_type", C.c_uint8),
        ("n_ref_frames", C.c_uint8),
        ("absrefdist", C.c_uint8 * 7),
        ("tile_rows", C.c_uint8),
        ("_pad1", C.c_uint8),
        ("tile_row_start_sb", C.c_uint16 * 65),
    ]


class FilmGrainData(C.Structure):
    _fields_ = [
        ("chroma_scaling_from_luma", C.c_int32),
        ("num_points", C.c_int32 * 3),
        ("points", ((C.c_uint8 * 2) * 14) * 3),
        ("scaling_shift", C.c_int32),
        ("ar_coeff_lag", C.c_int32),
        ("ar_coeffs", (C.c_int8 * 28) * 3),
        ("ar_coeff_shift", C.c_int32),
        ("grain_scale_shift", C.c_int32),
        ("uv_mult", C.c_int32 * 2),
        ("uv_luma_mult", C.c_int32 * 2),
        ("uv_offset", C.c_int32 * 2),
        ("overlap_flag", C.c_int32),
        ("clip_to_restricted_range", C.c_int32),
        ("mc_identity", C.c_int32),
        ("block_size", C.c_int32),
    ]


class SideInfo(C.Structure):
    _fields_ = [
        ("masks", C.c_void_p),
        ("lr", C.c_void_p),
        ("n_sb256", C.c_int32),
        ("segmap", C.c_void_p),
        ("segmap_stride", C.c_int32),
        ("segmap_uv", C.c_void_p),
        ("segmap_uv_stride", C.c_int32),
        ("db_masks", C.c_void_p),
    ]


# R2gDbBlock: one create_db_mask call (lf_mask.rs:399-503) of the decoder
DB_BLOCK_DTYPE = np.dtype([
    ("bx", "<u2"), ("by", "<u2"), ("bs", "u1"), ("flags", "u1"), ("tx_part", "u1"), ("seg_id", "u1"),
    ("inter_mode", "u1"), ("comp_type", "u1"), ("ref0", "i1"), ("ref1", "i1"),
])
DBB_CHROMA, DBB_INTRA, DBB_SKIP_TXFM, DBB_TX_LL, DBB_REFINE_MV = 1, 2, 4, 8, 16


class DbMaskInput(C.Structure):
    """R2gDbMaskInput: the frame's create_db_mask calls, the header fields
    subpu_flt_lvl reads (lf_mask.rs:367-397) and the tile starts that reset
    the edge-level contexts (decode.rs:207)."""
    _fields_ = [
        ("blocks", C.c_void_p),
        ("n_blocks", C.c_int32),
        ("sub_pu", C.c_uint8),
        ("tip_frame_mode", C.c_uint8),
        ("tip_subpel_filter", C.c_uint8),
        ("tip_refine_mv", C.c_uint8),
        ("n_tile_cols", C.c_int32),
        ("n_tile_rows", C.c_int32),
        ("tile_col_start4", C.c_uint16 * 64),
        ("tile_row_start4", C.c_uint16 * 64),
    ]


def db_mask_input(blocks, sub_pu=0, tip_frame_mode=0, tip_subpel_filter=0, tip_refine_mv=0,
                  tile_cols=(0,), tile_rows=(0,)):
    """Build an R2gDbMaskInput over a DB_BLOCK_DTYPE array (caller keeps it
    alive); tile starts in luma 4x4 units."""
    d = DbMaskInput()
    d.blocks = blocks.ctypes.data if len(blocks) else None
    d.n_blocks = len(blocks)
    d.sub_pu, d.tip_frame_mode, d.tip_subpel_filter, d.tip_refine_mv = sub_pu, tip_frame_mode, \
        tip_subpel_filter, tip_refine_mv
    d.n_tile_cols, d.n_tile_rows = len(tile_cols), len(tile_rows)
    for i, v in enumerate(tile_cols):
        d.tile_col_start4[i] = v
    for i, v in enumerate(tile_rows):
        d.tile_row_start4[i] = v
    return d


class BatchItem(C.Structure):
    _fields_ = [
        ("frame", C.c_void_p),
        ("fp", C.POINTER(FrameParams)),
        ("side", C.POINTER(SideInfo)),
        ("inloop_mask", C.c_uint32),
        ("fgd", C.POINTER(FilmGrainData)),
        ("grain_seed", C.c_uint32),
    ]


class ServeConfig(C.Structure):
    _fields_ = [("mem_budget", C.c_int64), ("max_batch", C.c_int32), ("frames_per_stream", C.c_int32)]


class ServeRequest(C.Structure):
    _fields_ = [
        ("stream_id", C.c_int32),
        ("fp", C.POINTER(FrameParams)),
        ("side", C.POINTER(SideInfo)),
        ("inloop_mask", C.c_uint32),
        ("fgd", C.POINTER(FilmGrainData)),
        ("grain_seed", C.c_uint32),
        ("src_y", C.c_void_p), ("src_u", C.c_void_p), ("src_v", C.c_void_p),
        ("src_y_stride", C.c_int64), ("src_uv_stride", C.c_int64),
        ("dst_y", C.c_void_p), ("dst_u", C.c_void_p), ("dst_v", C.c_void_p),
        ("dst_y_stride", C.c_int64), ("dst_uv_stride", C.c_int64),
        ("ref_y", C.c_void_p), ("ref_u", C.c_void_p), ("ref_v", C.c_void_p),
    ]


class ServeResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("batch_frames", C.c_int32), ("queue_us", C.c_double),
                ("latency_us", C.c_double)]


class ServeStats(C.Structure):
    _fields_ = [
        ("completed", C.c_int64), ("failed", C.c_int64), ("batches", C.c_int64),
        ("mean_batch", C.c_double), ("mpix", C.c_double),
        ("p50_us", C.c_double), ("p99_us", C.c_double), ("mean_us", C.c_double), ("max_us", C.c_double),
        ("span_s", C.c_double), ("issue_s", C.c_double),
        ("evictions", C.c_int64), ("resident_bytes", C.c_int64), ("pending", C.c_int64),
    ]


class WienerParamsSingle(C.Structure):
    """R2gWienerParamsSingle (WienerParamsSingle, looprestoration.rs:1716-1726)."""
    _fields_ = [("filter", C.c_void_p), ("luma", C.c_void_p), ("luma_top", C.c_void_p),
                ("luma_bottom", C.c_void_p), ("stride", C.c_int64), ("ss_ver", C.c_int32), ("ss_hor", C.c_int32),
                ("ds_flt", C.c_int32)]


class WienerParamsMulti(C.Structure):
    """R2gWienerParamsMulti (WienerParamsMulti, looprestoration.rs:1728-1734)."""
    _fields_ = [("filters", C.c_void_p), ("subclass_lut", C.c_void_p), ("noskip_mask", C.c_void_p),
                ("base_q", C.c_int32)]


class WienerParams(C.Union):
    """R2gWienerParams (WienerParamsC, looprestoration.rs:1736-1740)."""
    _fields_ = [("single", WienerParamsSingle), ("multi", WienerParamsMulti)]


# order of r2g_struct_sizes()
STRUCT_SIZES = [
    ("R2gAv2Filter", AV2_FILTER_DTYPE.itemsize),
    ("R2gAv2RestorationUnit", LR_UNIT_DTYPE.itemsize),
    ("R2gAv2Restoration", AV2_RESTORATION_DTYPE.itemsize),
    ("R2gFrameParams", C.sizeof(FrameParams)),
    ("R2gFilmGrainData", C.sizeof(FilmGrainData)),
    ("R2gSideInfo", C.sizeof(SideInfo)),
    ("R2gBatchItem", C.sizeof(BatchItem)),
    ("R2gServeConfig", C.sizeof(ServeConfig)),
    ("R2gServeRequest", C.sizeof(ServeRequest)),
    ("R2gServeResult", C.sizeof(ServeResult)),
    ("R2gServeStats", C.sizeof(ServeStats)),
    ("R2gWienerParams", C.sizeof(WienerParams)),
    ("R2gDbBlock", DB_BLOCK_DTYPE.itemsize),
    ("R2gDbMaskInput", C.sizeof(DbMaskInput)),
]


def plane_geometry(width, height, bitdepth):
    """Reference DefaultPicAllocator geometry (picture.rs:79-97), strides in bytes."""
    hbd = 1 if bitdepth > 8 else 0
    aw = (width + 127) & ~127
    ah = (height + 127) & ~127
    y_stride = aw << hbd
    uv_stride = y_stride >> 1
    if y_stride & 1023 == 0:
        y_stride += 64
    if uv_stride & 1023 == 0:
        uv_stride += 64
    return y_stride, uv_stride, ah, ah >> 1


def side_info(masks, lr, segmap=None, segmap_stride=0, segmap_uv=None, segmap_uv_stride=0, db_masks=None):
    """Build an R2gSideInfo pointing at numpy arrays (caller keeps them alive);
    `db_masks` is an optional DbMaskInput (kept alive by the caller too)."""
    s = SideInfo()
    s.db_masks = C.addressof(db_masks) if db_masks is not None else None
    s.masks = masks.ctypes.data
    s.lr = lr.ctypes.data
    s.n_sb256 = int(masks.shape[0])
    s.segmap = segmap.ctypes.data if segmap is not None else None
    s.segmap_stride = segmap_stride
    s.segmap_uv = segmap_uv.ctypes.data if segmap_uv is not None else None
    s.segmap_uv_stride = segmap_uv_stride
    return s
