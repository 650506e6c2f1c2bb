/*
 * oxideav_h266_b200.h — C ABI of the B200-native H.266/VVC in-loop filter chain.
 *
 * The chain is the decoder's picture-level filter stage, in the crate's order:
 * LMCS inverse luma map -> deblocking -> SAO -> ALF (+ CC-ALF).  Every entry
 * point mirrors one function of the Rust crate oxideav-h266 (v0.0.8) and takes
 * the same data, restated as plain C structs: sample planes are u16 row-major
 * with a stride, CU records are in decode order, CTB parameter arrays are in
 * raster CTB order.  Results are bit-exact with the crate's CPU filters.
 *
 * Memory: a picture's plane pointers are either host pointers
 * (H266_MEM_HOST: the call copies the planes to the device and back) or
 * device pointers on the context's device (H266_MEM_DEVICE: filtered in
 * place on the context's stream).  Side information (CU lists, CTB arrays,
 * APS tables) is always passed in host memory.
 *
 * Errors: every function returns H266_OK (0) or a negative H266_ERR_* code
 * and never aborts; h266_last_error() returns a message for the calling
 * thread's last failure.  The crate's filter functions are infallible and
 * panic on malformed input; here malformed input is rejected up front.
 *
 * Threading: a context is used by one thread at a time.  Calls on different
 * contexts may run concurrently.
 */
#ifndef OXIDEAV_H266_B200_H
#define OXIDEAV_H266_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define H266_OK 0
#define H266_ERR_INVALID_ARGUMENT (-1)
#define H266_ERR_GRID_MISMATCH (-2)    /* CTB array dims != picture CTB grid   */
#define H266_ERR_LMCS_CONFORMANCE (-3) /* derive_lmcs rejected the payload      */
#define H266_ERR_OUT_OF_MEMORY (-4)    /* device allocation failed              */
#define H266_ERR_TIMEOUT (-5)          /* a bounded device wait expired         */
#define H266_ERR_CUDA (-6)             /* any other CUDA runtime failure        */
#define H266_ERR_UNSUPPORTED (-7)      /* input outside the supported subset    */
#define H266_ERR_NO_DEVICE (-8)        /* no usable CUDA device                 */

/* ---- constants (src/aps.rs:21-33, src/lmcs.rs:42) ---------------------- */
#define H266_NUM_ALF_FILTERS 25
#define H266_ALF_LUMA_NUM_COEFF 12
#define H266_ALF_CHROMA_NUM_COEFF 6
#define H266_ALF_CC_NUM_COEFF 7
#define H266_ALF_MAX_CHROMA_ALT 8
#define H266_ALF_MAX_CC_FILTERS 4
#define H266_LMCS_NUM_BINS 16
/* DeblockCu::qp_c sentinel selecting the legacy QpY + offset arm
 * (src/deblock.rs:366-368, DEBLOCK_QP_C_LEGACY). */
#define H266_DEBLOCK_QP_C_LEGACY INT32_MIN

typedef enum h266_mem_kind { H266_MEM_HOST = 0, H266_MEM_DEVICE = 1 } h266_mem_kind;

/* ---- picture buffers (src/reconstruct.rs:41-52, 112-145) --------------- */
typedef struct h266_plane {
    uint16_t *samples;  /* row-major, stride * height samples                */
    uint64_t stride;    /* samples per row, >= width                          */
    uint32_t width;     /* visible width in samples                           */
    uint32_t height;    /* visible height in samples                          */
    uint32_t bit_depth; /* 8..16                                              */
    uint32_t reserved;
} h266_plane;

/* PictureBuffer: 4:2:0 luma + two chroma planes of the same bit depth. */
typedef struct h266_picture {
    h266_plane luma, cb, cr;
    uint32_t mem; /* h266_mem_kind of all three sample pointers */
    uint32_t reserved;
} h266_picture;

/* ---- deblocking (src/deblock.rs:52-161, 330-394) ----------------------- */
typedef struct h266_tb_split { /* TbSplit, src/deblock.rs:127-149 */
    uint8_t vertical;
    uint8_t n_bounds; /* 1..3 */
    uint8_t luma_only;
    uint8_t reserved0;
    uint32_t bounds[3];
    uint8_t y_coded[4];
    uint8_t cb_coded[4];
    uint8_t cr_coded[4];
} h266_tb_split;

typedef struct h266_tu64_cbf_map { /* Tu64CbfMap, src/deblock.rs:156-161 */
    uint8_t y[2][2];               /* [tile_y][tile_x] */
    uint8_t cb[2][2];
    uint8_t cr[2][2];
} h266_tu64_cbf_map;

typedef struct h266_deblock_cu { /* DeblockCu, src/deblock.rs:52-122 */
    uint32_t x, y, w, h;
    int32_t qp_y;
    int32_t qp_c[3]; /* [QpCb, QpCr, QpCbCr]; qp_c[0] == H266_DEBLOCK_QP_C_LEGACY -> legacy arm */
    uint8_t intra, tu_y_coded, tu_cb_coded, tu_cr_coded;
    uint8_t bdpcm_luma, bdpcm_chroma, plt, joint_cbcr2;
    uint8_t ciip, ibc, has_num_sb, has_tu64;
    uint8_t has_tb_split, reserved[3];
    uint32_t num_sb_x, num_sb_y; /* num_sb = Some((x, y)) when has_num_sb */
    h266_tu64_cbf_map tu64;      /* tu64 = Some(..) when has_tu64 */
    h266_tb_split tb_split;      /* tb_split = Some(..) when has_tb_split */
} h266_deblock_cu;

typedef struct h266_deblock_mv_cell { /* DeblockMvCell, src/deblock.rs:329-337 */
    uint8_t pred_l0, pred_l1, reserved[2];
    int32_t poc_l0, poc_l1;
    int32_t mv_l0[2], mv_l1[2]; /* 1/16 luma sample units */
} h266_deblock_mv_cell;

typedef struct h266_deblock_mv_grid { /* DeblockMvGrid, src/deblock.rs:344-348 */
    const h266_deblock_mv_cell *cells;
    uint64_t cells_w, cells_h;
} h266_deblock_mv_grid;

typedef struct h266_deblock_params { /* DeblockParams, src/deblock.rs:375-393 */
    uint32_t disabled;
    int32_t luma_beta_offset_div2, luma_tc_offset_div2;
    int32_t cb_beta_offset_div2, cb_tc_offset_div2;
    int32_t cr_beta_offset_div2, cr_tc_offset_div2;
    int32_t chroma_qp_offset_cb, chroma_qp_offset_cr;
    uint32_t bit_depth;
    uint32_t ctb_log2_size_y;
} h266_deblock_params;

/* ---- SAO (src/sao.rs:53-340) ------------------------------------------- */
typedef struct h266_sao_ctb { /* SaoCtb, src/sao.rs:134-144 */
    uint8_t sao_type_idx;     /* 0 not applied, 1 band offset, 2 edge offset */
    uint8_t eo_class;         /* 0 hor, 1 ver, 2 135deg, 3 45deg */
    uint8_t band_position;    /* 0..31 */
    uint8_t reserved;
    int32_t offset_val[5];    /* SaoOffsetVal after eq. 153; [0] == 0 */
} h266_sao_ctb;

typedef struct h266_sao_ctb_params { h266_sao_ctb luma, cb, cr; } h266_sao_ctb_params;

typedef struct h266_sao_picture { /* SaoPicture, src/sao.rs:211-217 */
    uint32_t pic_width_in_ctbs_y, pic_height_in_ctbs_y;
    const h266_sao_ctb_params *ctbs; /* raster CTB order */
} h266_sao_picture;

typedef struct h266_sao_config { /* SaoConfig, src/sao.rs:327-340 */
    uint32_t luma_used, chroma_used, bit_depth, ctb_log2_size_y, chroma_format_idc;
} h266_sao_config;

/* ---- ALF (src/alf.rs:67-206, src/aps.rs:77-102) ------------------------- */
typedef struct h266_alf_ctb { /* AlfCtb, src/alf.rs:66-87 */
    uint8_t luma_on, cb_on, cr_on;
    uint8_t luma_filt_set_idx; /* <16 fixed set, >=16 APS slot idx-16 */
    uint8_t cb_alt_idx, cr_alt_idx;
    uint8_t cc_cb_idc, cc_cr_idc; /* 0 off, k -> CC filter k-1 */
} h266_alf_ctb;

typedef struct h266_alf_picture { /* AlfPicture, src/alf.rs:90-96 */
    uint32_t pic_width_in_ctbs_y, pic_height_in_ctbs_y;
    const h266_alf_ctb *ctbs;
} h266_alf_picture;

typedef struct h266_alf_config { /* AlfConfig, src/alf.rs:136-158 */
    uint32_t alf_enabled, cb_enabled, cr_enabled, cc_cb_enabled, cc_cr_enabled;
    uint32_t bit_depth, ctb_log2_size_y, chroma_format_idc;
} h266_alf_config;

/* AlfApsData (src/aps.rs:77-102) with its Vec fields as fixed arrays plus
 * explicit lengths.  n_luma_filters must be 25 when the luma flag is set. */
typedef struct h266_alf_aps_data {
    uint8_t alf_luma_filter_signal_flag, alf_chroma_filter_signal_flag;
    uint8_t alf_cc_cb_filter_signal_flag, alf_cc_cr_filter_signal_flag;
    uint8_t alf_luma_clip_flag, alf_chroma_clip_flag, reserved[2];
    uint32_t alf_chroma_num_alt_filters_minus1;
    uint32_t n_luma_filters;   /* luma_coeff.len()  */
    uint32_t n_chroma_filters; /* chroma_coeff.len() (0..8) */
    uint32_t n_cc_cb_filters;  /* cc_cb_coeff.len() (0..4) */
    uint32_t n_cc_cr_filters;  /* cc_cr_coeff.len() (0..4) */
    int32_t luma_coeff[H266_NUM_ALF_FILTERS][H266_ALF_LUMA_NUM_COEFF];
    uint8_t luma_clip_idx[H266_NUM_ALF_FILTERS][H266_ALF_LUMA_NUM_COEFF];
    int32_t chroma_coeff[H266_ALF_MAX_CHROMA_ALT][H266_ALF_CHROMA_NUM_COEFF];
    uint8_t chroma_clip_idx[H266_ALF_MAX_CHROMA_ALT][H266_ALF_CHROMA_NUM_COEFF];
    int32_t cc_cb_coeff[H266_ALF_MAX_CC_FILTERS][H266_ALF_CC_NUM_COEFF];
    int32_t cc_cr_coeff[H266_ALF_MAX_CC_FILTERS][H266_ALF_CC_NUM_COEFF];
} h266_alf_aps_data;

typedef struct h266_alf_aps_binding { /* AlfApsBinding, src/alf.rs:179-195 */
    const h266_alf_aps_data *const *luma_apses; /* entries may be NULL (None) */
    uint32_t n_luma_apses;
    uint32_t reserved;
    const h266_alf_aps_data *chroma_aps; /* NULL = None */
    const h266_alf_aps_data *cc_cb_aps;
    const h266_alf_aps_data *cc_cr_aps;
} h266_alf_aps_binding;

/* ---- LMCS (src/lmcs.rs:50-153) ----------------------------------------- */
typedef struct h266_lmcs_data { /* LmcsData, src/lmcs.rs:50-76 */
    uint8_t lmcs_min_bin_idx, lmcs_delta_max_bin_idx, lmcs_delta_cw_prec_minus1;
    uint8_t lmcs_delta_abs_crs, lmcs_delta_sign_crs_flag, reserved[3];
    uint32_t lmcs_delta_abs_cw[H266_LMCS_NUM_BINS];
    uint8_t lmcs_delta_sign_cw_flag[H266_LMCS_NUM_BINS];
} h266_lmcs_data;

typedef struct h266_lmcs_derived { /* LmcsDerived, src/lmcs.rs:126-153 */
    uint32_t bit_depth, org_cw;
    uint32_t lmcs_cw[H266_LMCS_NUM_BINS];
    uint32_t input_pivot[H266_LMCS_NUM_BINS];
    uint32_t lmcs_pivot[H266_LMCS_NUM_BINS + 1];
    uint32_t scale_coeff[H266_LMCS_NUM_BINS];
    uint32_t inv_scale_coeff[H266_LMCS_NUM_BINS];
    int32_t lmcs_delta_crs;
    uint32_t chroma_scale_coeff[H266_LMCS_NUM_BINS];
} h266_lmcs_derived;

/* ---- whole chain (src/ctu.rs:11822-12065) ------------------------------- */
typedef struct h266_in_loop_filter_args {
    /* LMCS inverse map before deblocking (src/ctu.rs:11837-11851); NULL = off */
    const h266_lmcs_derived *lmcs;
    uint32_t lmcs_min_bin_idx, lmcs_max_bin_idx;
    /* deblocking inputs (src/ctu.rs:12006-12025) */
    const h266_deblock_cu *cus;
    uint64_t n_cus;
    const h266_deblock_cu *chroma_cus; /* NULL = share the luma records */
    uint64_t n_chroma_cus;
    const h266_deblock_mv_grid *mv_grid; /* NULL = None */
    h266_deblock_params deblock;
    uint32_t chroma_format_idc;
    uint32_t reserved0;
    const uint32_t *no_filter_cols;
    uint64_t n_no_filter_cols;
    const uint32_t *no_filter_rows;
    uint64_t n_no_filter_rows;
    /* SAO (src/ctu.rs:12026-12040); sao == NULL skips the pass */
    const h266_sao_picture *sao;
    h266_sao_config sao_cfg;
    uint32_t reserved1;
    /* ALF (src/ctu.rs:12046-12063); alf == NULL skips the pass */
    const h266_alf_picture *alf;
    h266_alf_config alf_cfg;
    const h266_alf_aps_binding *alf_binding;
    /* SAO / ALF clip bounds (0, gated lines..., extent); clip_cols == NULL = None */
    const uint32_t *clip_cols;
    uint64_t n_clip_cols;
    const uint32_t *clip_rows;
    uint64_t n_clip_rows;
} h266_in_loop_filter_args;

/* ---- context ------------------------------------------------------------ */
typedef struct h266_ctx h266_ctx;

/* Create a context on CUDA device `device` with its own stream and device
 * scratch.  Fails with H266_ERR_NO_DEVICE when the device is absent. */
int h266_ctx_create(int device, h266_ctx **out);
int h266_ctx_destroy(h266_ctx *ctx);
/* Use the caller's cudaStream_t (passed as void*) for later device work;
 * NULL restores the context's own stream. */
int h266_ctx_set_stream(h266_ctx *ctx, void *cuda_stream);
/* Block until all work queued on the context's stream has finished. */
int h266_ctx_synchronize(h266_ctx *ctx);
/* Message for the calling thread's last failed call ("" if none). */
const char *h266_last_error(void);
/* Number of kernels this context has launched since creation. */
uint64_t h266_ctx_kernel_launches(const h266_ctx *ctx);
/* Bytes of host -> device and device -> host copies the context has queued
 * for the chain calls (host picture planes and side information).  No
 * counterpart in the crate. */
int h266_ctx_transfer_bytes(const h266_ctx *ctx, uint64_t *h2d, uint64_t *d2h);

/* Per-kernel-family device time, for metrics and roofline accounting.  No
 * counterpart in the crate.  While profiling is on, every launch is bracketed
 * by CUDA events on the context's stream; h266_ctx_profile synchronizes the
 * stream, returns the accumulated milliseconds and launch counts per family
 * and resets them. */
#define H266_PROF_LMCS 0    /* LMCS LUT build and LUT-mapped plane copy      */
#define H266_PROF_DEBLOCK 1 /* deblocking edge-segment passes               */
#define H266_PROF_SAO_ALF 2 /* SAO / ALF / CC-ALF tile pass                 */
#define H266_PROF_COPY 3    /* plain plane copies into scratch              */
#define H266_PROF_FAMILIES 4
int h266_ctx_set_profiling(h266_ctx *ctx, int on);

/* Launch-shape tuning.  No counterpart in the crate.  The project's autotuner
 * (oxideav-h266_b200/autotune.py) sweeps these per picture geometry and bit
 * depth and persists the winners in a JSON table, which the Python layer
 * loads into a context with h266_ctx_set_tuning_for.  Keys and ranges:
 *   "e2e_group"            pictures per group of h266_apply_in_loop_filters_batch (1..16, default 4)
 *   "e2e_lanes"            slot sets (device buffers, a stream) those groups rotate over (1..16,
 *                          default 4)
 *   "sao_alf_ctas_per_sm"  SAO / ALF tile launches: 0 = one CTA per tile (default); 1..4 = a
 *                          persistent launch of that many CTAs per SM draining a device queue of
 *                          (picture, tile) items
 *   "sao_alf_tile_h"       SAO / ALF tile height for CTBs of 64 and 128: 64 (default) or 32
 *                          (values in between: 64)
 *   "prep_threads"         host threads preparing pictures' side information (0 = half the host
 *                          threads less two, 2..16; 1..64); a context-wide value
 *   "e2e_copy_streams"     1: every upload (planes, side information, batch tables) in issue order
 *                          on one stream and every download on another (default); 0: each group's
 *                          copies on its group's stream
 *   "e2e_ramp"             1: the batch starts and ends with groups of 1, 2, 4 ... pictures, so the
 *                          first kernels start and the last downloads end sooner (default); 0: all
 *                          groups of e2e_group pictures
 * h266_ctx_set_tuning sets the context's value; h266_ctx_set_tuning_for sets
 * it for batches whose largest picture has that luma size and bit depth, which
 * takes precedence.  Unknown keys or out-of-range values: H266_ERR_INVALID_ARGUMENT. */
int h266_ctx_set_tuning(h266_ctx *ctx, const char *key, int64_t value);
int h266_ctx_set_tuning_for(h266_ctx *ctx, uint32_t width, uint32_t height, uint32_t bit_depth, const char *key,
                            int64_t value);
int h266_ctx_get_tuning(const h266_ctx *ctx, const char *key, int64_t *value);
int h266_ctx_profile(h266_ctx *ctx, double ms[H266_PROF_FAMILIES], uint64_t launches[H266_PROF_FAMILIES]);
/* Host time of h266_apply_in_loop_filters_batch calls since the last call, in
 * milliseconds: [0] preparing pictures (summed over the worker threads),
 * [1] the issuing thread waiting for a preparation, [2] the issuing thread
 * issuing copies and launches.  Resets the counters. */
int h266_ctx_host_profile(h266_ctx *ctx, double ms[3]);

/* ---- filters ------------------------------------------------------------ */

/* LmcsData::derive / derive_lmcs (src/lmcs.rs:113, 302-404): the §7.4.3.19
 * derivations with every conformance check.  Host-only arithmetic.
 * Returns H266_ERR_LMCS_CONFORMANCE where the crate returns Err. */
int h266_derive_lmcs(const h266_lmcs_data *data, uint32_t bit_depth, h266_lmcs_derived *out);

/* Whole-plane LMCS inverse luma map, the loop at src/ctu.rs:11837-11851 over
 * LmcsDerived::idx_y_inv + inverse_map_luma_sample (src/lmcs.rs:209, 230). */
int h266_lmcs_inverse_map_luma(h266_ctx *ctx, h266_picture *pic, const h266_lmcs_derived *lmcs,
                               uint32_t lmcs_min_bin_idx, uint32_t lmcs_max_bin_idx);

/* Encoder chroma ALF decision: chroma_alf_decide_and_apply_clipped
 * (src/alf_enc.rs:628-821) for `component` 1 (Cb) or 2 (Cr).  One trial per
 * alternative filter of `aps` (every CTB on with that filter); per CTB the
 * option of lowest chroma SSE against `src` among {off, filter 0, ...} is kept
 * (earlier options win ties), its samples are written into rec's component
 * plane and apply_pic (the caller's AlfPicture records, n_apply = wc * hc,
 * host memory) gets cb_on / cb_alt_idx (or cr_*) for the chosen CTBs; other
 * records are left as they are.  No-op for chroma_format_idc 0 or an APS
 * without chroma filters, as in the crate.  Supported: 4:2:0, BitDepth
 * 8..14, coefficients in [-128, 127] (H266_ERR_UNSUPPORTED otherwise). */
int h266_chroma_alf_decide_and_apply_clipped(h266_ctx *ctx, const h266_picture *src, h266_picture *rec,
                                             h266_alf_ctb *apply_pic, uint64_t n_apply,
                                             const h266_alf_aps_data *aps, uint32_t component,
                                             uint32_t ctb_log2_size_y, uint32_t bit_depth,
                                             uint32_t chroma_format_idc, const uint32_t *col_bd,
                                             uint64_t n_col_bd, const uint32_t *row_bd, uint64_t n_row_bd);

/* Encoder CC-ALF decision: cc_alf_decide_and_apply_clipped (src/alf_enc.rs:
 * 935-1138).  As above with one trial per CC filter of `aps` for the
 * component (idc = filter + 1), each reading `pre_luma_alf` (the luma before
 * luma ALF, laid out as rec's luma plane, in rec->mem memory) and adding the
 * correction into rec's chroma; apply_pic gets cc_cb_idc (or cc_cr_idc). */
int h266_cc_alf_decide_and_apply_clipped(h266_ctx *ctx, const h266_picture *src, h266_picture *rec,
                                         const uint16_t *pre_luma_alf, h266_alf_ctb *apply_pic, uint64_t n_apply,
                                         const h266_alf_aps_data *aps, uint32_t component,
                                         uint32_t ctb_log2_size_y, uint32_t bit_depth, uint32_t chroma_format_idc,
                                         const uint32_t *col_bd, uint64_t n_col_bd, const uint32_t *row_bd,
                                         uint64_t n_row_bd);

/* Encoder SAO decision: sao_decide_picture (src/sao_enc.rs:385-487).  For
 * every CTB of rec's grid (luma size / CTB size rounded up), luma (when
 * sao_luma), Cb and Cr (when sao_chroma; Cr within Cb's type and class) get
 * the crate's band-offset / edge-offset choice from the src - rec statistics
 * of the CTB (4:2:0 chroma at half the luma CTB).  out: n_out = wc * hc
 * records in host memory; the pictures are not modified.  A sample above
 * (1 << bit_depth) - 1 has no band in the crate (its index runs out of
 * bounds) and makes the call return H266_ERR_INVALID_ARGUMENT. */
int h266_sao_decide_picture(h266_ctx *ctx, const h266_picture *src, const h266_picture *rec,
                            uint32_t ctb_log2_size_y, uint32_t bit_depth, uint32_t sao_luma, uint32_t sao_chroma,
                            h266_sao_ctb_params *out, uint64_t n_out);

/* Encoder chroma SAO merge: apply_chroma_sao_merge (src/sao_enc.rs:500-668).
 * In raster order every CTB of the independent SaoPicture (w_ctbs x
 * h_ctbs, raster records) keeps its own Cb/Cr parameters or takes those of
 * the already merged left / above CTB, whichever costs least (Cb + Cr SSE of
 * SAO on rec_pre_sao against src, plus 8 x the crate's bit estimate; earlier
 * options win ties).  merged: the resulting records (luma as given); map:
 * 0 independent, 1 merge left, 2 merge above.  Both outputs in host memory.
 * rec_pre_sao's Cb and Cr planes must have the same size and src's chroma
 * planes at least that size (the crate indexes them alike). */
int h266_sao_chroma_merge(h266_ctx *ctx, const h266_picture *src, const h266_picture *rec_pre_sao,
                          const h266_sao_ctb_params *independent, uint32_t w_ctbs, uint32_t h_ctbs,
                          uint32_t bit_depth, uint32_t ctb_log2_size_y, h266_sao_ctb_params *merged,
                          uint8_t *merge_map);
/* The same merge for n pictures at once (device pictures, H266_MEM_DEVICE):
 * each CTB anti-diagonal is one launch over the CTBs of every picture on it,
 * so the diagonals' few CTBs per picture fill the GPU together.  Per picture
 * i: srcs[i], pres[i], independent[i] (w_ctbs[i] x h_ctbs[i] records),
 * merged[i] and merge_maps[i] as for h266_sao_chroma_merge; results are the
 * same as n separate calls.  Returns when the results are in host memory. */
int h266_sao_chroma_merge_batch(h266_ctx *ctx, uint32_t n, const h266_picture *const *srcs,
                                const h266_picture *const *pres, const h266_sao_ctb_params *const *independent,
                                const uint32_t *w_ctbs, const uint32_t *h_ctbs, uint32_t bit_depth,
                                uint32_t ctb_log2_size_y, h266_sao_ctb_params *const *merged, uint8_t *const *merge_maps);

/* ---- recon-side LMCS (src/lmcs.rs:169-290, src/ctu.rs:734-742, 1701-1815) */
typedef struct h266_rect {
    uint32_t x, y, w, h;
} h266_rect;

/* CtuWalker::lmcs_forward_map_luma_rect (src/ctu.rs:1701-1727) over a list of
 * rectangles, in list order: every luma sample of each rectangle (clipped to
 * the plane) becomes Clip1(forward_map_luma_sample(s)) (src/lmcs.rs:186-194,
 * eq. 1213).  A sample inside k rectangles is mapped k times, as in the
 * crate's loop.  The crate has no bin for a sample above (1 << BitDepth) - 1
 * (its table index runs out of bounds): such a sample makes the call return
 * H266_ERR_INVALID_ARGUMENT.  Waits for the context stream. */
int h266_lmcs_forward_map_luma_rects(h266_ctx *ctx, h266_picture *pic, const h266_lmcs_derived *lmcs,
                                     const h266_rect *rects, uint64_t n_rects);

typedef struct h266_lmcs_cvs_block { /* one CU's eq. 1216 inputs (src/ctu.rs:1752-1815) */
    uint32_t x_cu_cb, y_cu_cb; /* luma origin of the CU holding the sizeY-aligned corner */
    uint8_t avail_l, avail_t;  /* nb_in_region() of the left / top neighbour; the
                                  picture-edge tests x_cu_cb > 0, y_cu_cb > 0 are applied here */
    uint8_t reserved[2];
} h266_lmcs_cvs_block;

/* CtuWalker::lmcs_chroma_var_scale_for_cu (src/ctu.rs:1752-1815) from the CU
 * origin and neighbour availability on, for n CUs: invAvgLuma over the left
 * column / top row of the (mapped) luma plane, sizeY = min(ctb_size_y, 64)
 * samples each with the crate's edge clamps (eqs. 1216/1217), idx_y_inv
 * (src/lmcs.rs:209-221) and ChromaScaleCoeff (eq. 1218).  var_scale: n
 * entries in host memory. */
int h266_lmcs_chroma_var_scale(h266_ctx *ctx, const h266_picture *pic, const h266_lmcs_derived *lmcs,
                               uint32_t lmcs_min_bin_idx, uint32_t lmcs_max_bin_idx, uint32_t ctb_size_y,
                               const h266_lmcs_cvs_block *blocks, uint64_t n, uint32_t *var_scale);

#define H266_NO_VAR_SCALE 0xFFFFFFFFu
typedef struct h266_chroma_res_block { /* one chroma TB of the inter residual add */
    uint32_t x, y, w, h;  /* chroma samples; x + w <= width, y + h <= height */
    uint32_t plane;       /* 1 = Cb, 2 = Cr */
    uint32_t var_scale;   /* eq. 1218 varScale, H266_NO_VAR_SCALE = none (the crate's None) */
    uint64_t res_offset;  /* index of the TB's first residual in `res` (row-major, w per row) */
} h266_chroma_res_block;

/* The inter chroma residual add (src/ctu.rs:9912-9945): each TB's residual,
 * folded by lmcs_scale_chroma_residuals (src/ctu.rs:734-742, eqs. 1219/1220)
 * when it has a varScale, is added to the plane with Clip1, TB by TB in list
 * order (overlapping TBs add in order).  `res` is host memory for
 * H266_MEM_HOST pictures and device memory for H266_MEM_DEVICE ones.  Waits
 * for the context stream. */
int h266_lmcs_add_chroma_residual(h266_ctx *ctx, h266_picture *pic, uint32_t bit_depth, const int32_t *res,
                                  uint64_t n_res, const h266_chroma_res_block *blocks, uint64_t n);

/* ---- output conversion (examples/decode_dump.rs, src/stream.rs:47-66) ---- */
typedef struct h266_crop_window { /* DecodedPicture::crop (src/stream.rs:59-61), luma samples */
    uint32_t left, top, width, height;
} h266_crop_window;

/* The cropped planar dump of a decoded picture as examples/decode_dump.rs:
 * 24-40 writes it (the bytes tests/jvet_conformance.rs:402-427 hash per
 * plane): luma rows, then, when chroma_format_idc != 0, Cb and Cr rows with
 * the crop window halved; one byte per sample (`v as u8`) when bit_depth <= 8,
 * else two bytes little-endian.  dst (dst_mem: H266_MEM_HOST or
 * H266_MEM_DEVICE) must hold the whole dump; *written receives its size
 * (dst == NULL: only the size, nothing is converted). */
int h266_output_convert(h266_ctx *ctx, const h266_picture *pic, const h266_crop_window *crop,
                        uint32_t chroma_format_idc, uint32_t bit_depth, void *dst, uint64_t dst_capacity,
                        uint32_t dst_mem, uint64_t *written);

/* apply_deblocking_clipped (src/deblock.rs:497-617). chroma_cus may be NULL
 * (None), mv_grid may be NULL (None). */
int h266_apply_deblocking_clipped(h266_ctx *ctx, h266_picture *pic, const h266_deblock_cu *cus,
                                  uint64_t n_cus, const h266_deblock_cu *chroma_cus,
                                  uint64_t n_chroma_cus, const h266_deblock_mv_grid *mv_grid,
                                  const h266_deblock_params *params, uint32_t chroma_format_idc,
                                  const uint32_t *no_filter_cols, uint64_t n_no_filter_cols,
                                  const uint32_t *no_filter_rows, uint64_t n_no_filter_rows);

/* apply_sao_clipped (src/sao.rs:389-497). col_bd == NULL means no tile bounds. */
int h266_apply_sao_clipped(h266_ctx *ctx, h266_picture *pic, const h266_sao_picture *sao_pic,
                           const h266_sao_config *cfg, const uint32_t *col_bd, uint64_t n_col_bd,
                           const uint32_t *row_bd, uint64_t n_row_bd);

/* apply_alf_clipped (src/alf.rs:235-434), CC-ALF included. */
int h266_apply_alf_clipped(h266_ctx *ctx, h266_picture *pic, const h266_alf_picture *alf_pic,
                           const h266_alf_config *cfg, const h266_alf_aps_binding *binding,
                           const uint32_t *col_bd, uint64_t n_col_bd, const uint32_t *row_bd,
                           uint64_t n_row_bd);

/* Encoder luma ALF decision: alf_decide_and_apply_clipped (src/alf_enc.rs:
 * 185-322) when aps == NULL, alf_decide_and_apply_with_aps_clipped
 * (src/alf_enc.rs:352-528) otherwise.  Trials 0..15 are the fixed filter sets
 * and trial 16 the APS set (APS slot 0); for every CTB the option of lowest
 * luma SSE against `src` among {off, trial 0, ...} is kept (earlier options win
 * ties), its samples are written into rec's luma plane (chroma untouched) and
 * decisions[] receives the returned AlfPicture (wc * hc entries, wc/hc =
 * rec luma size / CTB size rounded up; only luma_on and luma_filt_set_idx are
 * set).  sse, when not NULL, receives the per-CTB table
 * [off, trial 0, ..., trial T-1] (T = 16, or 17 with an APS) of uint64 sums.
 * Supported: BitDepth 8..14, CtbLog2SizeY 5..7, APS coefficients in
 * [-128, 127] (H266_ERR_UNSUPPORTED otherwise). */
int h266_alf_decide_and_apply_clipped(h266_ctx *ctx, const h266_picture *src, h266_picture *rec,
                                      const h266_alf_aps_data *aps, uint32_t ctb_log2_size_y,
                                      uint32_t bit_depth, uint32_t chroma_format_idc,
                                      const uint32_t *col_bd, uint64_t n_col_bd, const uint32_t *row_bd,
                                      uint64_t n_row_bd, h266_alf_ctb *decisions, uint64_t n_decisions,
                                      uint64_t *sse);

/* CtuWalker::apply_in_loop_filters_with_alf (src/ctu.rs:11822-12065) after its
 * gate lists are built: LMCS inverse -> deblock -> SAO -> ALF in one call. */
int h266_apply_in_loop_filters(h266_ctx *ctx, h266_picture *pic, const h266_in_loop_filter_args *args);

/* Batched form of h266_apply_in_loop_filters: n independent pictures (any mix
 * of sizes and bit depths) filtered by shared launches.  No counterpart in
 * the crate, which filters one picture per call (src/stream.rs:768). */
int h266_apply_in_loop_filters_batch(h266_ctx *ctx, uint32_t n, h266_picture *const *pics,
                                     const h266_in_loop_filter_args *const *args);

/* ---- resident plans ------------------------------------------------------
 * A plan holds one picture's filter side information on the device (deblock
 * edge segments, CTB parameter and APS tables, LMCS LUT) plus its scratch
 * planes, so the chain can run again on new samples with no host work.  No
 * counterpart in the crate, which rebuilds everything per call
 * (src/ctu.rs:11822-12065); the encoder's repeated ALF trials
 * (src/alf_enc.rs:244-1055) and a serving loop that keeps per-stream state
 * resident are the users.  `pic` gives only the plane sizes and bit depth at
 * create time; execute takes device planes of exactly that geometry and runs
 * asynchronously on the context's stream. */
typedef struct h266_chain_plan h266_chain_plan;
int h266_chain_plan_create(h266_ctx *ctx, const h266_picture *pic, const h266_in_loop_filter_args *args,
                           h266_chain_plan **out);
int h266_chain_plan_execute(h266_ctx *ctx, h266_chain_plan *plan, h266_picture *pic);
/* As h266_chain_plan_create, with flags.  H266_PLAN_DEVICE_SIDEINFO: the plan
 * keeps the CU lists, motion and no-filter lines instead of the derived edge
 * segments, and every execution derives the deblocking side information on
 * the device first (the CU map and edge walk of apply_deblocking_clipped,
 * src/deblock.rs:630-983, the work the crate does on every call), batched
 * over the pictures of h266_chain_plan_execute_batch.  Pictures the device
 * walk does not take (h266_sideinfo_mode 0: CUs off the 4x4 grid, outside the
 * picture or overlapping, a luma CU list with chained edges out of decode
 * order) keep host-derived segments, as without the flag. */
#define H266_PLAN_DEVICE_SIDEINFO 1u
int h266_chain_plan_create_ex(h266_ctx *ctx, const h266_picture *pic, const h266_in_loop_filter_args *args,
                              uint32_t flags, h266_chain_plan **out);
/* 1 when the plan derives its side information on the device at every
 * execution, 0 when it holds host-derived segments. */
int h266_chain_plan_device_sideinfo(const h266_chain_plan *plan);
/* Which deblocking side information a picture gets (host only, no context,
 * no device): 0 built on the host (the crate's walk, src/deblock.rs:630-983);
 * 1 built on the device, no two edge footprints can overlap (luma CUs and
 * transform blocks of at least 8 samples, no sub-block grids, 4:2:0 or 4:0:0:
 * the grid-mode tile kernel when SAO or ALF runs); 2 built on the device with
 * footprints that may chain, other chroma formats (the grid-mode strip
 * kernels).  Negative: an H266_ERR_* code for invalid arguments. */
int h266_sideinfo_mode(const h266_picture *pic, const h266_in_loop_filter_args *args);
/* Executes n plans on n device pictures (pics[i] with plans[i]; sizes may
 * differ) as one batch: one deblocking launch and one SAO / ALF launch per
 * kernel variant cover the tiles of every picture, so the GPU's tail between
 * pictures disappears.  No counterpart in the crate.  Asynchronous on the
 * context's stream, like h266_chain_plan_execute; results are bit-identical
 * to executing the plans one by one.  A picture must not appear twice. */
int h266_chain_plan_execute_batch(h266_ctx *ctx, uint32_t n, h266_chain_plan *const *plans,
                                  h266_picture *const *pics);
int h266_chain_plan_destroy(h266_chain_plan *plan);
/* A batched plan execution captured once into a CUDA graph and replayed with
 * one launch.  No counterpart in the crate.  The graph holds the batch's
 * parameter tables and refers to the plans and the pictures' device buffers
 * as they were at create time: a replay filters whatever samples those
 * buffers then hold, with the plans' side information; plans and buffers must
 * outlive the graph.  Replays go on the context's stream and are
 * bit-identical to h266_chain_plan_execute_batch on the same inputs.  The
 * context's tuning at create time is baked in. */
typedef struct h266_batch_graph h266_batch_graph;
int h266_batch_graph_create(h266_ctx *ctx, uint32_t n, h266_chain_plan *const *plans, h266_picture *const *pics,
                            h266_batch_graph **out);
int h266_batch_graph_launch(h266_ctx *ctx, h266_batch_graph *graph);
int h266_batch_graph_destroy(h266_batch_graph *graph);

/* Served filter chain: a request loop for many concurrent streams.  No
 * counterpart in the crate, which filters one picture per call on the
 * decoding thread (src/stream.rs:768).  Callers (any thread) submit a plan and
 * a device picture of its geometry; the server admits queued requests into a
 * batch whenever one of its three batch slots is free and the requests in
 * flight fit `memory_budget` (a request counts its picture's planes plus its
 * plan's scratch planes; an idle server always admits one), and runs the
 * batch as h266_chain_plan_execute_batch does on the slot's own stream, so
 * batches overlap on the GPU.  max_batch = 1 gives plain per-picture launches.
 * The server owns a context on `device`.  A picture must not be submitted
 * again before its request completed.  wait blocks until the request is done
 * and returns its status and its latency from submission to completion. */
typedef struct h266_server h266_server;
int h266_server_create(int device, uint32_t max_batch, uint64_t memory_budget, h266_server **out);
int h266_server_submit(h266_server *server, h266_chain_plan *plan, h266_picture *pic, uint64_t *ticket);
int h266_server_wait(h266_server *server, uint64_t ticket, double *latency_ms);
int h266_server_stats(h266_server *server, uint64_t *requests, uint64_t *batches);
/* Replays a request trace against the server from native threads: request i
 * (plans[i] on pics[i]) is submitted arrival_s[i] seconds after the call
 * starts (non-decreasing), and not before request after[i] (< i, or -1; NULL
 * for none) has completed -- the caller's picture-buffer reuse.  Returns when
 * every request is done, with latency_ms[i] = completion - scheduled arrival.
 * For load tests of a serving configuration. */
int h266_server_replay(h266_server *server, uint32_t n, h266_chain_plan *const *plans, h266_picture *const *pics,
                       const double *arrival_s, const int32_t *after, double *latency_ms);
/* A batch admits more than one request only while its pictures' luma samples
 * stay within `px` (default 1920 x 1080; 0: no cap), so a large picture does
 * not wait for a batch of smaller ones.  A batch of one request runs with
 * per-kernel launches, like h266_chain_plan_execute. */
int h266_server_set_batch_pixels(h266_server *server, uint64_t px);
int h266_server_destroy(h266_server *server); /* drains the queue first */

/* ---- allocation-free chain ---------------------------------------------------
 * No counterpart in the reference.  The whole chain (as h266_apply_in_loop_filters)
 * on device planes, for callers that cannot call cudaMalloc at run time:
 * real-time decode loops that ban allocator calls (and their unbounded latency)
 * once streaming starts, and hosts whose device memory all belongs to their own
 * pool, so a library allocation would fail or break their accounting.  The call
 * allocates no device memory: its scratch (side information, LMCS LUT,
 * deblocked planes) lives in one fixed device array of
 * H266_NOALLOC_SCRATCH_BYTES that every GPU loading the library keeps until the
 * process exits.  The caller passes the picture (H266_MEM_DEVICE planes,
 * filtered in place) and the stream (NULL = legacy default stream).
 *   - Pictures whose scratch need exceeds the array are rejected with
 *     H266_ERR_UNSUPPORTED and a message naming both sizes (1920x1080 4:2:0
 *     fits; 3840x2160 does not).
 *   - Every call looks up the array's device address on the current device
 *     (cudaGetSymbolAddress, which allocates nothing).
 *   - Every call builds the side information on the host and copies it from
 *     ordinary (pageable) host memory that is gone when the call returns, so
 *     the call cannot be recorded into a CUDA graph; graph replays of the
 *     chain are h266_batch_graph_create / h266_batch_graph_launch.
 *   - All calls share the one array and every call overwrites it: calls whose
 *     work overlaps on the GPU (other streams, other threads) race.  Serialize
 *     them on one stream.
 *   - Host-side side-information building still uses ordinary host memory. */
#define H266_NOALLOC_SCRATCH_BYTES (16u << 20)
int h266_apply_in_loop_filters_noalloc(h266_picture *pic, const h266_in_loop_filter_args *args, void *cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* OXIDEAV_H266_B200_H */
