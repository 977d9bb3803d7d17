/*
 * CPU oracle for the rav2d in-loop filter + film-grain path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a line-faithful C++ restatement of the
 * reference's scalar filter path (the rav2d Rust crate; every function cites
 * the file:line it follows, paths inside crates/rav2d/src).  It exists to
 * check the CUDA kernels: tests, the smoke check and the CPU-baseline leg of
 * the benchmark load it; the product library never links or calls it.
 *
 * It keeps the reference's per-superblock-row sequencing (deblock cols ->
 * rows -> copy_db -> CDEF(+CCSO) with the 8-row seam -> LR with its stripe
 * line buffers and left borders), so any quirk of that sequencing shows up
 * as a parity difference against the out-of-place GPU pipeline.
 *
 * Samples are stored as uint16_t for every bit depth; stores go through
 * pstore(), which wraps to the reference's storage width (u8 for 8-bit).
 */
#ifndef R2G_ORACLE_H
#define R2G_ORACLE_H

#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include <vector>

#include "rav2d_gpu.h"

namespace r2o {

typedef uint16_t pixel;

struct BD {
    int bitdepth;
    int bdmax() const { return (1 << bitdepth) - 1; }
    int bd8() const { return bitdepth - 8; }
    /* Pixel::from_i32 of the reference's storage type (pixel.rs:30-52). */
    pixel store(int v) const { return bitdepth == 8 ? (pixel)(uint8_t)v : (pixel)v; }
    int clip(int v) const { return v < 0 ? 0 : (v > bdmax() ? bdmax() : v); }
};

/* intops.rs */
static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline int iclip(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int apply_sign(int v, int s) { return s < 0 ? -v : v; }
static inline int ulog2(uint32_t v) { return 31 ^ __builtin_clz(v); }
static inline uint32_t uabs(int v) { return v < 0 ? (uint32_t)(-(int64_t)v) : (uint32_t)v; }

/* Layout constants (4:2:0 only). */
enum { SS_HOR = 1, SS_VER = 1 };

/* Frame-wide constant state, the shape of `LoopFilterState`
 * (internal.rs:152-230) plus `FilterFrameParams` (decode.rs:3645-3710). */
struct Frame {
    const R2gFrameParams *fp;
    BD bd;
    int hbd;  /* seq_hdr.hbd: 0 for 8-bit, 1 for 10-bit */
    int bw, bh; /* frame size in 4x4 units */
    int sbh, sb256w, sb256h;
    pixel *p[3];
    ptrdiff_t stride[2]; /* in samples */
    std::vector<R2gAv2Filter> mask; /* mutable copy (crop_bottom_edge) */
    const R2gAv2Restoration *lr_mask;
    const uint8_t *segmap;
    ptrdiff_t b4_stride;
    const uint8_t *segmap_uv;
    ptrdiff_t uv_segmap_stride;
    /* LoopFilterState derived scalars */
    int base_q, wiener_idx, ns_subclass_class_idx; /* -1 = None */
    int restore_planes, gdf_ref_dst_idx;
    std::vector<uint8_t> start_of_tile_row;
    /* line buffers */
    std::vector<pixel> lr_db_line[3];
    std::vector<pixel> cdef_line[2][3];
    int cdef_line_toggle;
};

/* deblock.cpp */
uint32_t deblock_quant_thr(int hbd, int qidx);
uint32_t deblock_side_thr(int hbd, int qidx);
int dq_lookup(int qidx);
int filter_choice(const pixel *buf, ptrdiff_t s, ptrdiff_t t, ptrdiff_t stride, int max_width_neg,
                  int max_width_pos, uint32_t q_thr, uint32_t side_thr);
void deblock_crop_bottom_edge(Frame &f, size_t mask_row, int sby);
void deblock_sbrow_cols(Frame &f, size_t mask_row, int sby);
void deblock_sbrow_rows(Frame &f, size_t mask_row, int sby);
void copy_db(Frame &f, int sby);
void backup_db(pixel *dst, const pixel *src, ptrdiff_t stride, int ss_ver, bool sb128, int row,
               int row_h, int w, bool lr_backup, int n_tc);

/* cdef.cpp */
int cdef_find_dir(const pixel *img, ptrdiff_t stride, uint32_t *var, int bd8);
int adjust_strength(int strength, uint32_t var);
int constrain(int diff, int threshold, int shift);
void cdef_filter_sbrow(Frame &f, size_t mask_row, int sby, uint32_t inloop);
uint32_t ccso_score(int diff, int quant_step, uint32_t edge_classifier);

/* lr.cpp */
int get_qval_given_tskip(int qstep, int tskip, int i, int bitdepth_min_8);
void lr_sbrow_apply(Frame &f, int sby, uint32_t inloop);

/* grain.cpp */
uint32_t get_random_number(uint32_t bits, uint32_t *state);
int round2(int x, uint32_t shift);
void generate_scaling(int bitdepth, const uint8_t (*points)[2], int num, uint8_t *scaling);

}  // namespace r2o

/* lf_mask.cpp: the decoder's walk over a frame's create_db_mask calls */
extern "C" void r2o_build_db_masks(const R2gDbMaskInput *in, const R2gFrameParams *fp, R2gAv2Filter *masks,
                                   int n_sb256);

#endif
