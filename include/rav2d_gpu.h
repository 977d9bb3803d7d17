/*
 * rav2d_gpu.h - C ABI of the B200 in-loop filter + film-grain library.
 *
 * This is the drop-in boundary for the post-reconstruction stage of the rav2d
 * AV2 decoder. A host decoder (the rav2d Rust crate through an `extern "C"`
 * FFI crate, or any C/C++/Python caller) keeps entropy decoding, prediction
 * and reconstruction on the CPU and hands each reconstructed frame plus its
 * filter side-info to this library, which runs deblocking, CDEF+CCSO, loop
 * restoration (NS-Wiener, PC-Wiener, GDF) and film grain on one GPU.
 *
 * Every struct below is a fixed-layout mirror of the reference's Rust types;
 * the citation on each gives the file:line (paths inside the rav2d project)
 * of the type it mirrors. Plain pointers and sizes only: no CUDA or torch
 * types appear in any signature.
 *
 * Sample storage: 8-bit frames are uint8_t samples, 10-bit frames uint16_t.
 * Strides are in BYTES, as in the reference's Picture (picture.rs:79-97).
 * Supported layout: 4:2:0, sb128 = 0, width and height multiples of 8, any
 * tile grid (several tile rows up to 128 superblock rows); anything else is
 * rejected with R2G_E_INVALID rather than filtered differently.
 *
 * Threading: a context is used by one host thread at a time. Calls enqueue
 * work on the context's streams and return; r2g_wait / r2g_sync block.
 */
#ifndef RAV2D_GPU_H
#define RAV2D_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference filters are infallible; these report
 * boundary misuse and device problems instead of aborting) ---- */
#define R2G_OK 0
#define R2G_E_INVALID (-1)  /* bad argument or unsupported configuration */
#define R2G_E_OOM (-2)      /* device-memory budget or allocation exhausted */
#define R2G_E_TIMEOUT (-3)  /* r2g_wait deadline passed; work still queued */
#define R2G_E_DEVICE (-4)   /* CUDA error or device-side watchdog tripped */
#define R2G_E_NOTREADY (-5) /* ticket not complete (non-blocking poll) */
#define R2G_E_TOO_LARGE (-6) /* request exceeds a fixed-size buffer's limit */

/* ---- inloop filter bitmask (looprestoration.rs:1697-1706) ---- */
#define R2G_INLOOP_DEBLOCK (1u << 0)
#define R2G_INLOOP_CDEF (1u << 1)
#define R2G_INLOOP_CCSO (1u << 2)
#define R2G_INLOOP_WIENER (1u << 3)
#define R2G_INLOOP_GDF (1u << 4)
#define R2G_INLOOP_ALL 0x1fu

/* ---- restoration types (looprestoration.rs:1671-1677) ---- */
#define R2G_RESTORE_NONE 0
#define R2G_RESTORE_PC_WIENER 1
#define R2G_RESTORE_NS_WIENER 2
#define R2G_RESTORE_SWITCHABLE 3

/* Per-SB256 filter side-info; mirrors `Av2Filter` (lf_mask.rs:8-19).
 * filter_y[dir][pos][k][i]: dir 0 = vertical edges (pos = x4 in the SB256,
 * i = sb64 row, bit = y4 in the sb64), dir 1 = horizontal edges (pos = y4,
 * i = sb64 column, bit = x4); k = edge class 0..3, k = 4 marks sub-PU edges.
 * filter_uv: the same for 4:2:0 chroma (pos = chroma x4/y4 in the SB256,
 * i = pair index, low/high byte for even/odd sb64).  sizeof == 12100. */
typedef struct R2gAv2Filter {
    uint16_t filter_y[2][64][5][4];
    uint16_t filter_uv[2][64][5][4];
    uint16_t qidx[16];
    uint8_t gdf[16];
    int8_t cdef_idx[16];
    uint8_t ccso[3];
    uint8_t _pad0;
    uint16_t noskip_mask[32][4];
    uint16_t lr_noskip_mask[64][4];
    uint16_t lossless_mask_y[64][4];
    uint16_t lossless_mask_uv[64][4];
} R2gAv2Filter;

/* Mirrors `Av2RestorationUnit` (lf_mask.rs:2-5).  sizeof == 513. */
typedef struct R2gAv2RestorationUnit {
    uint8_t restoration_type;
    int8_t ns_filter[16][32];
} R2gAv2RestorationUnit;

/* Mirrors `Av2Restoration` (lf_mask.rs:39-41): [plane][unit in SB256]. */
typedef struct R2gAv2Restoration {
    R2gAv2RestorationUnit lr[3][16];
} R2gAv2Restoration;

/* Mirrors `FhCcsoPlane` (headers.rs:640-652). */
typedef struct R2gCcsoPlane {
    uint8_t enabled;
    uint8_t bo_only;
    uint8_t scale_idx;
    uint8_t quant_idx;
    uint8_t ext_filter_support;
    uint8_t edge_clf;
    uint8_t max_band_log2;
    uint8_t _pad0;
    uint8_t filter_off[64];
} R2gCcsoPlane;

/* Mirrors `NSWienerPlane` + `FhRestorationPlane` (headers.rs:618-632). */
typedef struct R2gRestorationPlane {
    uint8_t restoration_type;
    uint8_t frame_filters_on;
    uint8_t num_classes_idx;
    uint8_t num_classes;
    int8_t filter[16][18];
} R2gRestorationPlane;

/* Frame-constant parameters of the filter path: the parts of the sequence
 * and frame headers that `FilterFrameParams::new` (decode.rs:3645-3710),
 * `init_wiener` (decode.rs:27), `compute_restore_planes` (decode.rs:59) and
 * `compute_gdf_ref_dst_idx` (decode.rs:67) read. */
typedef struct R2gFrameParams {
    int32_t width;  /* luma samples */
    int32_t height; /* luma samples */
    int32_t bitdepth; /* 8 or 10 */
    int32_t layout;   /* 1 = 4:2:0 (the only supported value) */
    int32_t sb128;    /* must be 0 */
    int32_t cfl_ds_filter_index; /* SequenceHeader.cfl_ds_filter_index */
    /* FhDeblock (headers.rs:590-598) */
    uint8_t deblock_level_y[2];
    uint8_t deblock_level_u;
    uint8_t deblock_level_v;
    int8_t deblock_delta_q_y[2];
    int8_t deblock_delta_q_u;
    int8_t deblock_delta_q_v;
    /* FhQuant (headers.rs:556-564): yac and the AC deltas */
    int32_t quant_yac;
    int8_t quant_uac_delta;
    int8_t quant_vac_delta;
    /* FhSegmentation (headers.rs:566-576): enabled, per-segment delta_q and
     * lossless flags.  segmap pointers may be NULL when disabled. */
    uint8_t seg_enabled;
    uint8_t _pad0;
    int16_t seg_delta_q[8];
    uint8_t seg_lossless[8];
    /* SequenceHeader.cdef + FhCdef (headers.rs:608-615) */
    uint8_t seq_cdef;
    uint8_t cdef_damping;
    uint8_t cdef_on_skiptx;
    uint8_t cdef_n_strengths;
    uint8_t cdef_y_strength[8];
    uint8_t cdef_uv_strength[8];
    /* FhCcso (headers.rs:673-677) */
    R2gCcsoPlane ccso[3];
    /* FhRestoration (headers.rs:634-638) */
    R2gRestorationPlane restoration[3];
    uint8_t restoration_unit_size[2]; /* log2, luma / chroma */
    /* FhGdf (headers.rs:601-606): enabled is AdaptiveBoolean (0 = off) */
    uint8_t gdf_enabled;
    uint8_t gdf_qp_idx;
    uint8_t gdf_scale;
    /* inputs of compute_gdf_ref_dst_idx: frame_type & 1 = inter/switch */
    uint8_t frame_type;
    uint8_t n_ref_frames;
    uint8_t absrefdist[7];
    /* TileInfo rows (headers.rs:325-337), read by init_start_of_tile_row
     * (decode.rs:99-120) for the loop-restoration stripes: tile_rows and
     * row_start_sb in superblock units (tile_rows + 1 entries).  tile_rows
     * 0 is taken as one tile row. */
    uint8_t tile_rows;
    uint8_t _pad1;
    uint16_t tile_row_start_sb[65];
} R2gFrameParams;

/* Mirrors `FilmGrainData` (headers.rs:509-525). */
typedef struct R2gFilmGrainData {
    int32_t chroma_scaling_from_luma;
    int32_t num_points[3];
    uint8_t points[3][14][2];
    int32_t scaling_shift;
    int32_t ar_coeff_lag;
    int8_t ar_coeffs[3][28];
    int32_t ar_coeff_shift;
    int32_t grain_scale_shift;
    int32_t uv_mult[2];
    int32_t uv_luma_mult[2];
    int32_t uv_offset[2];
    int32_t overlap_flag;
    int32_t clip_to_restricted_range;
    int32_t mc_identity;
    int32_t block_size;
} R2gFilmGrainData;

/* Opaque handles. */
typedef struct R2gCtx R2gCtx;
typedef struct R2gFrame R2gFrame;

/* Frame side-info as the reference keeps it in `LoopFilterState`
 * (internal.rs:152-167) after Phase A: n_sb256 = sb256w * sb256h masks in
 * raster order, the same count of restoration records, and the optional
 * segment maps (b4 granularity; NULL = all segment 0). */
struct R2gDbMaskInput;
typedef struct R2gSideInfo {
    const R2gAv2Filter *masks;
    const R2gAv2Restoration *lr;
    int32_t n_sb256;
    const uint8_t *segmap;
    int32_t segmap_stride;
    const uint8_t *segmap_uv;
    int32_t segmap_uv_stride;
    /* Optional (NULL = the masks' filter_y / filter_uv are used as given):
     * the deblock edge masks are built on the device from the decoder's
     * create_db_mask calls instead, and only the other Av2Filter fields
     * are uploaded (filter_y / filter_uv of `masks` are not read). */
    const struct R2gDbMaskInput *db_masks;
} R2gSideInfo;

/* One create_db_mask call of the decoder (decode.rs:7869-7912 for a coded
 * block, :12893-12928 for a TIP superblock; lf_mask.rs:399-503): the
 * Av2Block fields the mask builders read, for the luma call (bs, bx, by)
 * or the chroma call (cbs, cbx, cby) of the block.  sizeof == 12. */
typedef struct R2gDbBlock {
    uint16_t bx, by;     /* frame position in luma 4x4 units */
    uint8_t bs;          /* BlockSize (levels.rs) */
    uint8_t flags;       /* R2G_DBB_* */
    uint8_t tx_part;     /* TxPartition of the luma transform split */
    uint8_t seg_id;
    uint8_t inter_mode;  /* data.inter.inter_mode */
    uint8_t comp_type;   /* data.inter.comp_type */
    int8_t ref0, ref1;   /* ref_pair.r */
} R2gDbBlock;
#define R2G_DBB_CHROMA (1u << 0)    /* the chroma call (filter_uv) */
#define R2G_DBB_INTRA (1u << 1)     /* is_intra */
#define R2G_DBB_SKIP_TXFM (1u << 2) /* skip_txfm */
#define R2G_DBB_TX_LL (1u << 3)     /* tx_size_ll (lossless luma transform) */
#define R2G_DBB_REFINE_MV (1u << 4) /* data.inter.refine_mv */

/* The frame's create_db_mask calls with the header fields they read
 * (subpu_flt_lvl, lf_mask.rs:367-397) and the tile grid, whose starts reset
 * the edge-level contexts (decode.rs:207 reset_context: the left context at
 * every tile column of every superblock row, the above context at every
 * tile row).  Blocks may come in any order: a block's context is the level
 * its left / above neighbour left there, which is what the decoder's walk
 * (neighbours first) reads. */
typedef struct R2gDbMaskInput {
    const R2gDbBlock *blocks;
    int32_t n_blocks;
    uint8_t sub_pu;            /* frame_hdr.deblock.sub_pu */
    uint8_t tip_frame_mode;    /* frame_hdr.tip.frame_mode */
    uint8_t tip_subpel_filter; /* frame_hdr.tip.subpel_filter */
    uint8_t tip_refine_mv;     /* seq_hdr.tip_refine_mv */
    int32_t n_tile_cols, n_tile_rows;
    uint16_t tile_col_start4[64]; /* luma 4x4 units; [0] == 0, increasing */
    uint16_t tile_row_start4[64];
} R2gDbMaskInput;

/* ---- version / capability ---- */
int r2g_version(void);
/* Plane geometry of the reference's DefaultPicAllocator (picture.rs:79-97):
 * width/height aligned to 128, stride in bytes, bumped by 64 when it is a
 * multiple of 1024.  Pure host function. */
int r2g_plane_geometry(int width, int height, int bitdepth, int64_t *y_stride,
                       int64_t *uv_stride, int64_t *y_rows, int64_t *uv_rows);
/* Bytes of `sizeof` for each ABI struct, so a binding can check its mirror. */
int r2g_struct_sizes(int32_t *sizes, int n);

/* ---- context: one per host thread; `device` is the CUDA ordinal,
 * `mem_budget` the device bytes the context may hold (0 = no limit). ---- */
int r2g_ctx_create(int device, int64_t mem_budget, R2gCtx **out);
int r2g_ctx_destroy(R2gCtx *ctx);
const char *r2g_last_error(R2gCtx *ctx);
/* Enqueue the context's filter work on a caller-owned CUDA stream
 * (a cudaStream_t passed as void*; NULL restores the context's own stream). */
int r2g_ctx_set_stream(R2gCtx *ctx, void *stream);
/* Copy overlap (no counterpart in the reference, whose filters work on host
 * memory): when enabled, r2g_frame_upload_recon copies on an upload
 * stream, r2g_frame_stage on a second upload stream (its small side-info
 * copies then overlap the recon upload instead of queueing behind it) and
 * r2g_download on a download stream of the context, each frame's copies and
 * kernels ordered by events, so the transfers of one frame overlap the
 * kernels of another.  r2g_sync waits for all of these streams; r2g_ctx_fence makes the context stream wait for every copy issued
 * so far (an event recorded on it afterwards marks the end of all of them).
 * In this mode host buffers are read asynchronously: page-locked recon
 * planes, and side-info records that are page-locked (they are then copied
 * without staging), must stay unchanged until the frame's work completes.
 * Off by default: then every call runs on the context stream in order. */
int r2g_ctx_overlap_copies(R2gCtx *ctx, int enable);
int r2g_ctx_fence(R2gCtx *ctx);
/* Instrumentation (no counterpart in the reference): when enabled, every
 * r2g_frame_run / r2g_frame_grain records CUDA events between its kernels;
 * r2g_ctx_profile_read synchronises and returns per-stage milliseconds and
 * launch counts summed since enabling, for stages 0 deblock, 1 CDEF+CCSO,
 * 2 loop restoration, 3 film grain. */
int r2g_ctx_profile(R2gCtx *ctx, int enable);
int r2g_ctx_profile_read(R2gCtx *ctx, double *stage_ms, int64_t *stage_launches, int n);
/* Number of kernels this context has launched since creation. */
int64_t r2g_ctx_launch_count(R2gCtx *ctx);

/* ---- device-resident frames (frame buffers live in the context) ---- */
int r2g_frame_alloc(R2gCtx *ctx, int width, int height, int bitdepth, R2gFrame **out);
int r2g_frame_free(R2gCtx *ctx, R2gFrame *f);
/* Upload the reconstructed planes (host pointers, byte strides). */
int r2g_frame_upload_recon(R2gCtx *ctx, R2gFrame *f, const void *y, int64_t y_stride,
                           const void *u, const void *v, int64_t uv_stride);
/* Stage the frame's side-info on the device (validate, apply the bottom-edge
 * crop (applied by the deblock kernel), upload masks / restoration records /
 * segment maps) without running
 * any stage; r2g_frame_run then runs the stages on the staged side-info. */
int r2g_frame_stage(R2gCtx *ctx, R2gFrame *f, const R2gFrameParams *fp, const R2gSideInfo *side,
                    uint32_t inloop_mask);
/* Run the filter stages of a staged frame on its uploaded recon (the recon
 * buffer is left unchanged, so a staged frame can be run again). */
int r2g_frame_run(R2gCtx *ctx, R2gFrame *f);
/* Copy a staged frame's SB256 records back as the stage kernels read them
 * (with R2gSideInfo.db_masks: filter_y / filter_uv as the device built them
 * from the block records).  `n` must be the frame's SB256 count.  No
 * counterpart in the reference; for inspection and tests. */
int r2g_frame_read_masks(R2gCtx *ctx, R2gFrame *f, R2gAv2Filter *out, int n);
/* Run every enabled stage for the whole frame (r2g_frame_stage followed by
 * r2g_frame_run).  Equivalent to calling the
 * reference's `filter_sbrow` (decode.rs:3718-4058) for every sby of the frame
 * in order; replaces the Phase-B loop at decode.rs:3597-3625. */
int r2g_frame_filter(R2gCtx *ctx, R2gFrame *f, const R2gFrameParams *fp,
                     const R2gSideInfo *side, uint32_t inloop_mask);
/* Film grain on the filtered frame into the frame's display copy; replaces
 * `apply_grain_to_picture_mt` (decode.rs:4672). */
int r2g_frame_grain(R2gCtx *ctx, R2gFrame *f, const R2gFilmGrainData *fgd, uint32_t seed);
/* No counterpart in the reference (its filters cannot fail).  Waits for the
 * context's stream and returns in *count how many bounded device-side waits
 * of the stage kernels ran out (0 in a healthy run; a kernel whose wait ran
 * out stops its work item and leaves its output incomplete). */
int r2g_ctx_device_faults(R2gCtx *ctx, uint32_t *count);
/* Copy the filtered planes (which = 0) or the grained display copy
 * (which = 1) into host memory; enqueued, complete after r2g_sync. */
int r2g_download(R2gCtx *ctx, R2gFrame *f, int which, void *y, int64_t y_stride, void *u,
                 void *v, int64_t uv_stride);
/* Block until every call enqueued on the context has finished. */
int r2g_sync(R2gCtx *ctx);

/* ---- output formatting and partial downloads ----
 * r2g_download_y4m: one Y4M frame of the filtered (which 0) or grained
 * (which 1) picture into `dst`, as rav2d-cli's write_picture / pack_plane
 * and Y4mWriter::write_frame produce it (crates/rav2d-cli/src/main.rs:114-149,
 * y4m.rs:36-45): "FRAME\n" then the Y, U and V planes tightly packed,
 * 16-bit little-endian samples above 8 bits.  out_bitdepth 0 keeps the
 * frame's depth; 8 on a 10-bit frame reduces samples to 8 bits on the device
 * ((v + 2) >> 2, clipped; a display option the reference does not have).
 * The planes are packed by a kernel and copied back in one transfer;
 * dst_size must be at least r2g_y4m_frame_bytes(...).
 * r2g_y4m_header: the stream header line rav2d-cli writes (y4m.rs:17-31,
 * main.rs:98-111 colorspace tags) for a 4:2:0 stream; returns its length.
 * r2g_download_rows: rows [row0, row0 + nrows) of the luma plane and the
 * co-located chroma rows (row0 and nrows even), e.g. the band of a reference
 * frame that the next frame's reconstruction reads. */
int r2g_download_y4m(R2gCtx *ctx, R2gFrame *f, int which, int out_bitdepth, void *dst, int64_t dst_size);
int64_t r2g_y4m_frame_bytes(int width, int height, int out_bitdepth);
int r2g_y4m_header(int width, int height, int fps_num, int fps_den, int bitdepth, char *buf, int cap);
int r2g_download_rows(R2gCtx *ctx, R2gFrame *f, int which, int row0, int nrows, void *y, int64_t y_stride,
                      void *u, void *v, int64_t uv_stride);

/* ---- DSP-context slots (crates/rav2d/src/dsp.rs:9-122) ----
 * Per-block functions for the self-contained slots of the reference's
 * DSPContext, with the reference functions' argument meaning and order; the
 * reference declares these slots but never fills or calls them, and the
 * per-frame entry points above are the performance path.  Each call copies
 * the block and the neighbours the reference would read to the GPU, runs one
 * kernel and copies the result back, synchronously, on the current device:
 * on a non-blocking stream the library owns, so a call neither waits for nor
 * delays work queued on the caller's streams.  Calls are serialised with each
 * other (they share a small per-device scratch buffer, allocated on a
 * device's first DSP call).
 * Host buffers hold u8 samples at bitdepth 8, u16 above; strides count
 * samples.  `top` points at row -2 and `bottom` at row h (column 0) of the
 * block, both with the block's stride; `left` holds [h][2] samples (columns
 * -2, -1); edges: 1 left, 2 right, 4 top, 8 bottom available (CDEF_HAVE_*,
 * cdef.rs:6-9). */
/* DeblockDSPContext.deblock_sb (dsp.rs:86-89): deblock_{h,v}_sb64{y,uv}_bd
 * (deblock.rs:303-548), one 64-long edge of 16 four-line segments.  `dst`
 * is the first positive-side sample of line 0; vert != 0: a vertical edge
 * (lines run down the rows, the h variants), else horizontal.  vmask[4]:
 * edge-class bits per segment (class 3 only for luma), ll_mask[0] / [1]:
 * lossless negative / positive sides, q_thr[16] / side_thr[16] per segment,
 * `edge` clamps the negative side to 6 (luma) / 2 (chroma) samples. */
int r2g_dsp_deblock_sb64(void *dst, int64_t stride, const uint16_t *vmask, const uint16_t *ll_mask,
                         const uint16_t *q_thr, const uint16_t *side_thr, int edge, int luma, int vert,
                         int bitdepth);
/* FilmGrainDSPContext.fgy_32x32xn / fguv_32x32xn (dsp.rs:9-16):
 * filmgrain.rs:248-407 / :409-598 on one row band (bh rows, pw samples) of
 * the caller's planes: dst = src + noise, `in_seed` the frame's grain seed,
 * `row_num` the band index, `scaling` the plane's (1 << bitdepth)-entry LUT,
 * `grain_lut` its [73][82] template; for chroma `luma_row` / `luma_stride`
 * are the band's luma rows, uv 0 = U / 1 = V, sx / sy the subsampling.
 * Samples above the bit depth's range are rejected (R2G_E_INVALID). */
int r2g_dsp_fgy_32x32xn(void *dst, const void *src, int64_t stride, const R2gFilmGrainData *data,
                        uint32_t in_seed, int pw, const uint8_t *scaling, const int16_t *grain_lut, int bh,
                        int row_num, int bitdepth);
int r2g_dsp_fguv_32x32xn(void *dst, const void *src, int64_t stride, const R2gFilmGrainData *data,
                         uint32_t in_seed, int pw, const uint8_t *scaling, const int16_t *grain_lut, int bh,
                         int row_num, const void *luma_row, int64_t luma_stride, int uv, int is_id, int sx,
                         int sy, int bitdepth);
/* CdefDSPContext.dir: cdef_find_dir_bd (cdef.rs:134-216) on the 8x8 block at
 * img; returns the direction 0..7 (or < 0 on error), *var its variance. */
int r2g_dsp_cdef_dir(const void *img, int64_t stride, uint32_t *var, int bitdepth);
/* CdefDSPContext.fb[0..2]: cdef_filter_block (cdef.rs:320-458) in place on a
 * w x h block (8x8, 4x8 or 4x4) with cdef_padding's rules (cdef.rs:37-114). */
int r2g_dsp_cdef_filter(void *dst, int64_t stride, const void *left, const void *top, const void *bottom,
                        int pri, int sec, int dir, int damping, int w, int h, int edges, int bitdepth);
/* CcsoDSPContext.prep: ccso_prep (ccso.rs:115-187) of a w x h output block
 * whose co-located luma region (w << ss_hor) x (h << ss_ver) starts at src;
 * class / band indices into dst.  Region at most 64 x 32 luma samples. */
int r2g_dsp_ccso_prep(uint8_t *dst, int64_t dst_stride, const void *src, int64_t stride, const void *left,
                      const void *top, const void *bottom, int max_band_log2, int ext_filter, int quant_step,
                      int edge_clf, int bo_only, int edges, int w, int h, int ss_hor, int ss_ver, int bitdepth);
/* CcsoDSPContext.add: ccso_add (ccso.rs:215-254) in place; offset_idxs[64]
 * packed offset indices, offset_lut[8], ll_mask [h/4][4] lossless bits.
 * w, h multiples of 4, at most 64. */
int r2g_dsp_ccso_add(void *dst, int64_t dst_stride, const uint8_t *idx, int64_t idx_stride,
                     const uint8_t *offset_idxs, const int8_t *offset_lut, int w, int h, const uint16_t *ll_mask,
                     int bitdepth);
/* LoopRestorationDSPContext.gdf_add: the GdfAddFn slot (looprestoration.rs:
 * 1770-1779; gdf_add :273-329) in place on a w x h block, w, h <= 64. */
int r2g_dsp_gdf_add(void *p, int64_t stride, const int8_t *err, int64_t err_stride, int w, int h, int scale,
                    const uint16_t *ll_mask, int bitdepth);
/* WienerParamsC (looprestoration.rs:1716-1740): the per-call parameters of
 * the WienerFilterFn slots.  Sample pointers are u8 at bitdepth 8, u16
 * above; strides count samples. */
typedef struct R2gWienerParamsSingle {
    const int8_t *filter;    /* 16 taps (luma) or 6 + 12 taps (chroma) */
    const void *luma;        /* chroma: co-located pre-LR luma at the block origin */
    const void *luma_top;    /* chroma: the 2 saved deblocked luma rows above */
    const void *luma_bottom; /* chroma: the 2 saved deblocked luma rows below */
    int64_t stride;          /* luma stride */
    int32_t ss_ver, ss_hor, ds_flt;
} R2gWienerParamsSingle;
typedef struct R2gWienerParamsMulti {
    const void *filters;         /* NS multi: int8_t[class][18]; PC: int16_t[class][13] */
    const uint8_t *subclass_lut; /* PC_WIENER_LUT_TO_CLASS class -> filter class */
    const uint16_t *noskip_mask; /* one 16-bit row mask per 4 rows */
    int32_t base_q;
} R2gWienerParamsMulti;
typedef union R2gWienerParams {
    R2gWienerParamsSingle single;
    R2gWienerParamsMulti multi;
} R2gWienerParams;

/* LoopRestorationDSPContext.ns_wiener_single[0] / [1], .ns_wiener_multi,
 * .pc_wiener: the WienerFilterFn slot (looprestoration.rs:1742-1753;
 * ns_wiener_single_y :524, ns_wiener_single_uv :1145, ns_wiener_multi
 * :1061, pc_wiener :1102) in place on a w x h block of one stripe (w <= 64,
 * h <= 64, multiples of 4).  `left` holds [h][6] samples (the unit to the
 * left's pre-filter border), `top` the 2 saved deblocked rows above the
 * stripe (row -2 first, column 0, stride dst_stride), `bottom` the 2 below
 * (row h first); `ll_mask` [h/4 + 1][4] lossless 4x4 bits; edges as
 * LR_HAVE_* (1 left, 2 right, 4 top, 8 bottom). */
int r2g_dsp_ns_wiener_single_y(void *dst, int64_t dst_stride, const void *left, const void *top, const void *bottom,
                               int w, int h, const R2gWienerParams *params, int edges, const uint16_t *ll_mask,
                               int bitdepth);
int r2g_dsp_ns_wiener_single_uv(void *dst, int64_t dst_stride, const void *left, const void *top,
                                const void *bottom, int w, int h, const R2gWienerParams *params, int edges,
                                const uint16_t *ll_mask, int bitdepth);
int r2g_dsp_ns_wiener_multi(void *dst, int64_t dst_stride, const void *left, const void *top, const void *bottom,
                            int w, int h, const R2gWienerParams *params, int edges, const uint16_t *ll_mask,
                            int bitdepth);
int r2g_dsp_pc_wiener(void *dst, int64_t dst_stride, const void *left, const void *top, const void *bottom, int w,
                      int h, const R2gWienerParams *params, int edges, const uint16_t *ll_mask, int bitdepth);
/* LoopRestorationDSPContext.gdf_prep: the GdfPrepFn slot (looprestoration.rs:
 * 1755-1768; gdf_prep :1432-1640): the GDF error of every sample of the w x h
 * luma block at p (w, h <= 64, even) into dst, with the same left / top /
 * bottom conventions (6 left columns, 2 saved rows each side). */
int r2g_dsp_gdf_prep(int8_t *dst, int64_t dst_stride, const void *p, int64_t stride, const void *left,
                     const void *top, const void *bottom, int w, int h, int ref_dst_idx, int qp_idx, int edges,
                     int bitdepth);
/* FilmGrainDSPContext.generate_grain_y / generate_grain_uv[1] (filmgrain.rs:
 * 115-230, 4:2:0): the 82x73 luma template and the two 44x38 chroma templates
 * (top-left of 82x73 arrays); any buffer may be NULL. */
int r2g_dsp_generate_grain(int16_t *buf_y, int16_t *buf_u, int16_t *buf_v, const R2gFilmGrainData *fgd,
                           uint32_t seed, int bitdepth);

/* ---- one-call convenience: host recon in, host filtered/grained out ---- */
int r2g_filter_frame_host(R2gCtx *ctx, const R2gFrameParams *fp, const R2gSideInfo *side,
                          uint32_t inloop_mask, const R2gFilmGrainData *fgd, uint32_t grain_seed,
                          const void *src_y, const void *src_u, const void *src_v,
                          int64_t y_stride, int64_t uv_stride, void *dst_y, void *dst_u,
                          void *dst_v, void *grain_y, void *grain_u, void *grain_v);

/* ---- batching: one persistent launch per stage over many frames ---- */
typedef struct R2gBatchItem {
    R2gFrame *frame;
    const R2gFrameParams *fp;
    const R2gSideInfo *side;
    uint32_t inloop_mask;
    const R2gFilmGrainData *fgd; /* NULL = no grain */
    uint32_t grain_seed;
} R2gBatchItem;
/* Enqueue the whole batch (at most 1023 distinct frames) as one persistent
 * launch per stage; frames of at least 1.5 M luma samples (1080p and up),
 * which fill the GPU alone, run through the per-frame pipeline first, on
 * the same stream.  Returns a ticket for r2g_wait.  An item whose fp and side
 * are both NULL runs with the side-info of the frame's last r2g_frame_stage
 * (as r2g_frame_run does); its inloop_mask is then ignored.  Film grain is
 * applied per item when fgd is non-NULL (read it back with which = 1). */
int r2g_batch_submit(R2gCtx *ctx, const R2gBatchItem *items, int n, uint64_t *ticket);
/* Wait for a ticket; R2G_E_TIMEOUT after timeout_ms (<0 = forever),
 * timeout_ms == 0 polls (R2G_E_NOTREADY when pending). */
int r2g_wait(R2gCtx *ctx, uint64_t ticket, int timeout_ms);
/* ---- serving: continuous batching over many concurrent streams ----
 * No counterpart in the reference (its decoder filters one frame at a time
 * inside Decoder::decode_frame, decode.rs:3597-3625).  A server owns one
 * worker thread that admits queued frames under a device-memory budget,
 * keeps each stream's frame buffers and side-info resident on the device,
 * and issues every admitted frame in the next batch while earlier batches
 * run (uploads, kernels and downloads of consecutive batches overlap).
 * While a server is attached, drive its context only through the server. */
typedef struct R2gServer R2gServer;
typedef struct R2gServeConfig {
    int64_t mem_budget;        /* bytes for resident frames; 0 = the context budget (or none) */
    int32_t max_batch;         /* frames per batch, 1..1023 (0 = 64) */
    int32_t frames_per_stream; /* resident device frames per stream (0 = 2) */
} R2gServeConfig;
typedef struct R2gServeRequest {
    int32_t stream_id;
    const R2gFrameParams *fp; /* copied at submit */
    const R2gSideInfo *side;  /* the records it points to stay valid until r2g_server_wait */
    uint32_t inloop_mask;
    const R2gFilmGrainData *fgd; /* NULL = no grain; copied at submit */
    uint32_t grain_seed;
    /* recon planes (host; pinned memory lets the upload overlap compute) */
    const void *src_y, *src_u, *src_v;
    int64_t src_y_stride, src_uv_stride; /* bytes */
    /* display output (grained when fgd, else filtered) */
    void *dst_y, *dst_u, *dst_v;
    int64_t dst_y_stride, dst_uv_stride; /* bytes; also used for ref_* */
    /* optional: the filtered (reference) frame as well; NULL = skip */
    void *ref_y, *ref_u, *ref_v;
} R2gServeRequest;
typedef struct R2gServeResult {
    int32_t status;       /* R2G_OK, or the error that failed this frame */
    int32_t batch_frames; /* frames in the batch it ran in */
    double queue_us;      /* submit -> issued */
    double latency_us;    /* submit -> output in host memory */
} R2gServeResult;
typedef struct R2gServeStats {
    int64_t completed, failed, batches;
    double mean_batch, mpix;
    double p50_us, p99_us, mean_us, max_us;
    double span_s;  /* first submit -> last completion */
    double issue_s; /* worker time spent enqueuing */
    int64_t evictions, resident_bytes, pending;
} R2gServeStats;
int r2g_server_create(R2gCtx *ctx, const R2gServeConfig *cfg, R2gServer **out);
/* Queue one frame; any thread.  Returns its id for r2g_server_wait. */
int r2g_server_submit(R2gServer *s, const R2gServeRequest *req, uint64_t *id);
/* Wait for a frame (timeout_ms < 0: forever; 0: poll -> R2G_E_NOTREADY;
 * R2G_E_TIMEOUT when it runs out).  On R2G_OK `res` holds the frame's own
 * status and the id is released. */
int r2g_server_wait(R2gServer *s, uint64_t id, int timeout_ms, R2gServeResult *res);
/* Free a stream's resident frames once its queued frames have completed. */
int r2g_server_close_stream(R2gServer *s, int32_t stream_id);
/* Latency / throughput statistics since creation or the last reset. */
int r2g_server_stats(R2gServer *s, R2gServeStats *st, int reset);
/* Completes every queued frame, then stops the worker and frees all. */
int r2g_server_destroy(R2gServer *s);

/* Instrumentation (no counterpart in the reference): the grid the last
 * batch used for stages 0 deblock, 1 CDEF+CCSO, 2 loop restoration, 3 film
 * grain (autotuned): CTAs per SM of a persistent grid, or 0 for one CTA per
 * work item; returns the SM count. */
int r2g_batch_config(R2gCtx *ctx, int32_t *ctas_per_sm, int n);

/* Instrumentation (no counterpart in the reference): the tile shape the last
 * batch used per stage, as luma rows per work item (deblock 64, CDEF+CCSO 32,
 * loop restoration 32 or 16 as autotuned, film grain the grain block size or
 * 0 without grain); returns the number of stages written. */
int r2g_batch_tile_rows(R2gCtx *ctx, int32_t *rows, int n);

/* ---- film grain without any device allocation ----
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * a decoder embedded in a framework whose device memory is owned by that
 * framework's allocator or a fixed pool, or a latency-critical output thread
 * that must not block in the driver's allocator.  Applies the same film grain
 * as r2g_frame_grain from the caller's device planes src_* (filtered frame,
 * 4:2:0) to the caller's device planes dst_* (display copy), byte strides,
 * enqueued on `stream` (a cudaStream_t; NULL = the legacy default stream).
 * Allocates nothing: its only scratch (grain templates and scaling LUTs, 40 KB)
 * is a fixed device array that every GPU loading the library holds until the
 * process exits.  The first call on a device (with that device current) looks
 * up the array's address and should come before any stream capture.  All
 * calls share the array, so calls whose GPU work overlaps race; serialise
 * them (one stream).  Bit depths above 10 exceed the array's LUT capacity and
 * return R2G_E_TOO_LARGE; other bad arguments (including film-grain fields
 * outside the ranges the reference's parser admits) return R2G_E_INVALID.
 * The array's address is looked up once per device and kept for the life of
 * the process: the library does not support cudaDeviceReset between calls. */
int r2g_film_grain_apply_noalloc(const void *src_y, const void *src_u, const void *src_v, void *dst_y,
                                 void *dst_u, void *dst_v, int64_t y_stride, int64_t uv_stride, int width,
                                 int height, int bitdepth, const R2gFilmGrainData *fgd, uint32_t seed,
                                 void *stream);

#ifdef __cplusplus
}
#endif

#endif /* RAV2D_GPU_H */
