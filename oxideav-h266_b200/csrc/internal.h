// Internal declarations shared by the CUDA translation units of the filter
// chain library (not part of the C ABI).
#pragma once

#include <cuda.h>  // CUtensorMap (the driver entry point is fetched at run time; nothing links libcuda)
#include <cuda_runtime.h>

#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "oxideav_h266_b200.h"

namespace h266 {

// ---------------------------------------------------------------- errors
struct Status {
  int code = H266_OK;
  bool ok() const { return code == H266_OK; }
};
int set_error(int code, const std::string &msg);  // records msg for h266_last_error, returns code
int cuda_error(cudaError_t e, const char *what);   // H266_ERR_CUDA (or OUT_OF_MEMORY) with context
#define H266_CUDA(call)                                   \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_error(e_, #call);  \
  } while (0)
#define H266_TRY(call)          \
  do {                          \
    int rc_ = (call);           \
    if (rc_ != H266_OK) return rc_; \
  } while (0)

// ---------------------------------------------------------------- host worker pool
// Fixed set of host threads that run the items of one job at a time
// (fn(0) .. fn(n-1), in any order and in parallel).  The thread that starts a
// job may wait for single items, so it can consume results in order while the
// workers are still producing later ones.  One job at a time per pool.
class TaskPool {
 public:
  explicit TaskPool(unsigned threads);
  ~TaskPool();
  TaskPool(const TaskPool &) = delete;
  TaskPool &operator=(const TaskPool &) = delete;
  unsigned size() const { return (unsigned)workers_.size(); }
  void start(size_t n, std::function<void(size_t)> fn);  // returns at once
  void wait_item(size_t i);                               // item i of the current job has finished
  void wait_all();                                        // every item of the current job has finished
  void run(size_t n, std::function<void(size_t)> fn) {    // start + wait_all
    start(n, std::move(fn));
    wait_all();
  }

 private:
  void loop();
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable work_cv_, done_cv_;
  std::function<void(size_t)> fn_;
  std::vector<uint8_t> done_;
  size_t n_ = 0, next_ = 0, finished_ = 0;
  bool stop_ = false;
};

// ---------------------------------------------------------------- device buffers
// A growable device allocation owned by a context.
struct DevBuf {
  void *ptr = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes);
  void release();
  template <class T>
  T *as() const {
    return static_cast<T *>(ptr);
  }
};

// A device plane view used by the kernels.
struct DPlane {
  uint16_t *s;
  int64_t stride;  // samples
  int w, h;
};

// ---------------------------------------------------------------- deblocking
// One edge segment of the reference's deblocking walk: a 4-line luma or a
// 2-line chroma piece of a vertical or horizontal edge.  (x, y) is q0 of the
// segment's first line in the plane's own sample grid.
struct EdgeSeg {
  uint16_t x, y;
  uint16_t beta, tc;
  uint8_t plane;  // 0 luma, 1 cb, 2 cr
  uint8_t bs;
  uint8_t mfl;    // mfl_p << 4 | mfl_q
  uint8_t flags;  // bit0 vertical, bit1 ctb_row (luma EDGE_HOR CTB row), bit2 plt_p, bit3 plt_q
};
static_assert(sizeof(EdgeSeg) == 12, "EdgeSeg layout");

// Host-side deblocking plan: segments grouped into independent components.
// Segments of one component touch overlapping samples and are listed in the
// reference's processing order; different components touch disjoint samples.
struct DeblockPlan {
  std::vector<EdgeSeg> segs[2];      // [0] vertical pass, [1] horizontal pass
  std::vector<uint32_t> comp[2];     // component start offsets (+ final end)
  uint32_t max_comp_len[2] = {0, 0};
  // per (plane, pass) lists before concatenation, index plane * 2 + pass; each
  // on its own cache lines, as different threads fill them
  struct alignas(64) Part {
    std::vector<EdgeSeg> segs;
    std::vector<uint32_t> comp;
    uint32_t max_len = 0;
  };
  Part parts[6];
  // Band index of each pass for the strip kernels, planes concatenated:
  // band_first[d][band_off[d][p] + b] is the first component of plane p's band
  // b and the plane's n_bands[d][p] + 1-th entry ends its last band.  Bands
  // are 4 luma / 2 chroma rows (vertical pass) or columns (horizontal pass);
  // components of bands beyond the plane touch no sample and are left out.
  std::vector<uint32_t> band_first[2];
  uint32_t band_off[2][3] = {{0, 0, 0}, {0, 0, 0}};
  uint32_t n_bands[2][3] = {{0, 0, 0}, {0, 0, 0}};
  // Component ranges of the tile kernel (kDeblockTile x kDeblockTile luma
  // tiles and the co-located chroma tiles).  Inside a band the components are
  // sorted and disjoint, so those reaching one tile form a range: for the
  // vertical pass tile_bounds[tb_off[0][p] + (band * tiles_x + tx) * 2] and the
  // next entry are the first and end component of the band reaching tile
  // column tx; for the horizontal pass the same with (column band * tiles_y +
  // ty).  tiles_ok is false when a component spans more than the tile halo, a
  // tile would list more components than the kernel's shared list holds, or
  // the chroma format is not 4:2:0 / 4:0:0; the strip kernels run then.
  bool tiles_ok = false;
  uint32_t tiles_x = 0, tiles_y = 0;
  std::vector<uint32_t> tile_bounds;
  uint32_t tb_off[2][3] = {{0, 0, 0}, {0, 0, 0}};
};

constexpr int kDeblockTile = 64;      // luma tile edge of the tile kernel
constexpr int kDeblockHaloY = 16;     // luma halo (a component's footprint is at most 16 samples)
constexpr int kDeblockHaloC = 8;      // chroma halo (footprints of at most 8 samples)
constexpr int kTileListY = 320;       // shared list entries per pass: luma components of a tile
constexpr int kTileListC = 176;       // chroma components of a tile, per plane

int build_deblock_plan(const h266_picture &pic, const h266_deblock_cu *cus, uint64_t n_cus,
                       const h266_deblock_cu *chroma_cus, uint64_t n_chroma, const h266_deblock_mv_grid *mv,
                       const h266_deblock_params &params, uint32_t cfi, const uint32_t *nf_cols, uint64_t n_cols,
                       const uint32_t *nf_rows, uint64_t n_rows, DeblockPlan &plan, TaskPool *pool = nullptr);

// Launches the two deblocking passes (vertical then horizontal) in place on
// the three device planes.  seg/comp point at device copies of the plan.
// Strip kernels: the vertical pass on row bands read from `src` (luma mapped
// through `lut` when given) and written to `dst` (which may be `src`), then the
// horizontal pass on 16-column strips of `dst` in place.
bool deblock_strips_fit(const DPlane planes[3]);
struct StripSide {  // device pointers of one pass
  const EdgeSeg *segs;
  const uint32_t *comp;
  const uint32_t *band_first;
};
int launch_deblock_strips(cudaStream_t st, const DPlane src[3], const DPlane dst[3], const uint16_t *lut,
                          int bit_depth, const StripSide &v, const StripSide &h, const uint32_t band_off[2][3],
                          const uint32_t n_bands[2][3], uint64_t *launches);
// Tile kernel: both passes per tile, from `src` (luma through `lut` when
// given) into `dst`, which must not overlap `src`.
int launch_deblock_tiles(cudaStream_t st, const DPlane src[3], const DPlane dst[3], const uint16_t *lut,
                         int bit_depth, const StripSide &v, const StripSide &h, const uint32_t *tile_bounds,
                         const uint32_t tb_off[2][3], const uint32_t n_bands[2][3], uint32_t tiles_x,
                         uint32_t tiles_y, uint64_t *launches);
// Batched tile kernel: fill_deblock_tile_params writes one picture's kernel
// parameters (deblock_tile_params_size() bytes) to `out` and returns its CTA
// count; CTAs [first[i], first[i + 1]) of the batched launch are picture i's.
size_t deblock_tile_params_size();
uint32_t fill_deblock_tile_params(void *out, const DPlane src[3], const DPlane dst[3], const uint16_t *lut,
                                  int bit_depth, const StripSide &v, const StripSide &h, const uint32_t *tile_bounds,
                                  const uint32_t tb_off[2][3], const uint32_t n_bands[2][3], uint32_t tiles_x,
                                  uint32_t tiles_y);
int launch_deblock_tiles_batch(cudaStream_t st, const void *d_params, const uint32_t *d_first, int n, uint32_t ctas,
                               uint64_t *launches);
// ---------------------------------------------------------------- device-built side information
// Device-built side information: the edge walk runs on the device from the
// CU lists and the motion grid and writes each segment to a dense per-band
// cell grid.  device_walk_mode returns 1 when no two segments' footprints can
// overlap (luma CUs and transform blocks at least 8 samples, no sub-block
// edges, 4:2:0 or 4:0:0): every cell is a component and the tile kernel scans
// the grids; 2 when footprints may chain (the strip kernels run each band's
// runs of cells in position order, which needs the luma CU list in decode
// order along every row and column of its CU map); 0 when the host must build
// the plan (CUs off the 4x4 grid, outside the picture or overlapping, CU lists
// out of order, planes too large for the strip kernels, invalid input).
int device_walk_mode(const h266_picture &pic, const h266_deblock_cu *cus, uint64_t n_cus,
                     const h266_deblock_cu *chroma_cus, uint64_t n_chroma, const h266_deblock_params &params,
                     uint32_t cfi);
// The CU lists travel to the device packed: per CU its first kCuHeadBytes
// (position, size, QPs, flags, sub-block counts), and a CuTail (the 64-sample
// TU map and TB split) only for CUs that have either; with motion by CU, a
// CuMotionRec only for CUs that are not intra (intra CUs read no motion).
// The walk's first launch expands them into full records in its scratch.
constexpr size_t kCuHeadBytes = 56;
static_assert(offsetof(h266_deblock_cu, tu64) == kCuHeadBytes, "CU head layout");
static_assert(sizeof(h266_deblock_cu) == kCuHeadBytes + 40, "CU tail layout");
// The compact head (16 bytes) used when every CU of a list fits it: 16-bit
// position and size, 8-bit QPs (qp_c[0] -128: the legacy sentinel, the other
// two then unused), the CU's flags as bits (every use of them is boolean),
// 8-bit sub-block counts.
struct CuCompact {
  uint16_t x, y, w, h;
  int8_t qp_y, qp_c[3];
  uint16_t flags;  // bit order: intra, tu_y/cb/cr_coded, bdpcm_luma/chroma, plt, joint_cbcr2, ciip, ibc,
                   // has_num_sb, has_tu64, has_tb_split
  uint8_t nsb_x, nsb_y;
};
static_assert(sizeof(CuCompact) == 16, "compact CU head");
struct CuTail {
  uint32_t index;
  uint8_t tail[40];  // bytes [kCuHeadBytes, sizeof(h266_deblock_cu)) of the CU
};
struct CuMotionRec {
  uint32_t index;
  h266_deblock_mv_cell m;
};
struct DeviceWalkIn {  // device pointers
  const uint8_t *heads[2];  // packed CU heads: luma list, chroma list (== heads[0] for a single tree)
  bool compact[2];          // the list's heads are CuCompact records (else kCuHeadBytes each)
  const CuTail *tails[2];
  uint64_t n_tails[2];
  uint64_t n_cus, n_chroma;
  bool sep;                              // a separate chroma tree
  const h266_deblock_mv_cell *mv_cells;  // nullptr: no motion grid (or motion by CU)
  uint64_t mv_w, mv_h;
  const CuMotionRec *mv_recs;  // motion by luma CU (every CU's cells agree): the non-intra CUs' records
  uint64_t n_mv_recs;
  bool mv_by_cu;
  const uint32_t *nf_cols, *nf_rows;
  uint64_t n_cols, n_rows;
  h266_deblock_params params;
  uint32_t cfi;
  int w, h, cw, ch;      // luma and chroma plane sizes
  uint32_t max_cu_dim;   // largest width or height of the CUs with edges inside them (4: none);
                         // the walk launches offsets 0 .. max_cu_dim - 4 (step 4)
  bool tile_lists;       // also list each tile's cells for the grid-mode tile kernel
  bool tiles_consume;    // the tile kernel (not the strip kernels) reads the grids: empty cells need no clearing
};
size_t device_walk_bytes(const DeviceWalkIn &in);  // scratch for the CU maps and segment grids
struct DeviceWalkOut {
  EdgeSeg *grid[2][3];
  uint32_t slots[2][3], bands[2][3];
  uint32_t tiles_x, tiles_y;
  uint32_t *tile_count;       // with DeviceWalkIn::tile_lists: cells per (tile, pass, plane)
  uint32_t *tile_list[2][3];  // and their grid indices, kTileListY / kTileListC per tile
};
int launch_device_walk(cudaStream_t st, const DeviceWalkIn &in, uint8_t *scratch, DeviceWalkOut &out,
                       uint64_t *launches);
int launch_deblock_tiles_grid(cudaStream_t st, const DPlane src[3], const DPlane dst[3], const uint16_t *lut,
                              int bit_depth, const DeviceWalkOut &g, uint64_t *launches);
int launch_deblock_strips_grid(cudaStream_t st, const DPlane src[3], const DPlane dst[3], const uint16_t *lut,
                               int bit_depth, const DeviceWalkOut &g, uint64_t *launches);
// Batched device walk: fill_walk_batch_item writes one picture's item
// (walk_batch_item_size() bytes) and its CTA counts per launch; the prefix
// sums of those counts over the batch's pictures (n + 1 entries each) select
// the picture of a CTA.  The three launches clear the pictures' scratch, build
// the CU maps and walk the edges; the grid-mode tile parameters of each
// picture then go into a batched tile launch like any other.
struct WalkBatchCounts {
  uint32_t clear_ctas = 0, grid_ctas = 0, walk_ctas = 0, offsets = 0;  // offsets: the largest, over the batch
};
size_t walk_batch_item_size();
void fill_walk_batch_item(void *out, const DeviceWalkIn &in, uint8_t *scratch, DeviceWalkOut &g, WalkBatchCounts &c);
int launch_walk_batch(cudaStream_t st, const void *d_items, const uint32_t *d_first_clear,
                      const uint32_t *d_first_grid, const uint32_t *d_first_walk, int n, const WalkBatchCounts &total,
                      uint64_t *launches);
uint32_t fill_deblock_tile_params_grid(void *out, const DPlane src[3], const DPlane dst[3], const uint16_t *lut,
                                       int bit_depth, const DeviceWalkOut &g);
int launch_deblock(cudaStream_t st, const DPlane planes[3], int bit_depth, const EdgeSeg *d_segs_v,
                   const uint32_t *d_comp_v, uint32_t n_comp_v, const EdgeSeg *d_segs_h, const uint32_t *d_comp_h,
                   uint32_t n_comp_h, uint64_t *launches);

// ---------------------------------------------------------------- LMCS
int derive_lmcs(const h266_lmcs_data *d, uint32_t bd, h266_lmcs_derived *o);
// Builds the 65536-entry inverse-map LUT on the device (one entry per u16 input).
int launch_lmcs_lut(cudaStream_t st, uint16_t *d_lut, const h266_lmcs_derived &l, uint32_t mn, uint32_t mx,
                    uint64_t *launches);
// dst = lut ? lut[src] : src over a plane (dst may equal src).
int launch_plane_map(cudaStream_t st, DPlane dst, DPlane src, const uint16_t *d_lut, uint64_t *launches);

// ---------------------------------------------------------------- SAO / ALF
struct SaoCtbDev {  // one component's SAO parameters for one CTB
  uint8_t type, eo_class, band_pos, pad;
  int16_t off[4];   // SaoOffsetVal[1..4]
};
struct CtbDev {      // everything pass 2 needs per CTB
  SaoCtbDev sao[3];  // 36 bytes
  uint16_t rect[4];  // SAO / ALF clip rectangle, luma samples (x0, y0, x1, y1)
  int16_t luma_set;  // ALF luma filter set slot, -1 = luma ALF off
  int8_t chroma_filt[2];  // chroma ALF alt filter per cb/cr, -1 = off
  int8_t cc_filt[2];      // CC-ALF filter per cb/cr, -1 = off
  int8_t pad[2];
};
static_assert(sizeof(CtbDev) == 52, "CtbDev layout");

struct AlfTablesDev {
  // luma filter sets: slot -> [25 classes][12] coefficients and clip values
  const int32_t *luma_coeff;  // slot s at [s * 600, s * 600 + 300)
  const int32_t *luma_clip;   // slot s at [s * 600, s * 600 + 300) (resolved AlfClip values)
  int32_t chroma_coeff[8][6];
  int32_t chroma_clip[8][6];
  int32_t cc_coeff[2][4][7];  // [cb/cr][filter][tap]
  // packed-arithmetic form (sao_alf2.cu): per tap three words (c|c<<16, -c|-c<<16, coeff & 0xff)
  const uint32_t *luma_packed;  // [slot][class * 4 + transposeIdx][12 taps][3], taps pre-permuted
  uint32_t chroma_packed[8 * 18];  // [alt][6 taps][3]
};

struct Pass2Args {
  // TMA descriptors of the three input planes (2-D u16 tensors, the tile
  // kernel's window boxes); valid when `tma` is set.  First, for the 64-byte
  // alignment the TMA unit needs.
  CUtensorMap tmap[3];
  int tma;        // windows staged by TMA (else 16-byte vector loads)
  int tile_h;     // tile height for CTBs of 64 and 128: 64 (also 0) or 32
  int sao_i8;     // every SAO offset of the picture fits a signed byte (the packed offset tables)
  DPlane src[3];  // input planes (post-deblock)
  DPlane dst[3];  // output planes
  int bit_depth;
  int ctb_log2;
  int sub_w, sub_h;       // chroma subsampling of the SAO / ALF config
  int chroma;             // chroma planes present (cfi != 0 and non-empty)
  int w_ctbs, h_ctbs;     // CTB parameter grid
  int tiles_x, tiles_y;   // 32x32 luma tiles
  int ext_w, ext_h;       // luma extent the tile grid covers
  int pic_w, pic_h;       // luma picture dims
  int has_clip;           // tile / slice clip bounds given
  // SAO
  int sao_luma, sao_chroma;
  // ALF
  int alf_luma_any, alf_chroma_cb, alf_chroma_cr, alf_cc_cb, alf_cc_cr;
  const CtbDev *ctbs;
  AlfTablesDev tables;
};

int launch_pass2(cudaStream_t st, const Pass2Args &a, bool do_sao, bool do_alf, uint64_t *launches);
// Fills a.tmap / a.tma for the packed tile kernel's windows of a.src (plane
// bases 16-byte aligned, strides multiples of 8 samples; otherwise a.tma = 0
// and the kernel loads its windows itself).  Host only, allocates nothing.
void pass2_tma_maps(Pass2Args &a);
// A 2-D tensor map of plane p with a box_w x box_h box (u16 samples, zero
// fill outside the plane); false when the plane's base or stride is not
// 16-byte aligned or the driver entry point is missing.
bool encode_plane_map(CUtensorMap *m, const DPlane &p, int box_w, int box_h);
// Deblocking tiles whose region copies timed out since the last call (read and cleared).
int deblock_wait_timeouts(uint32_t *count);
// Timeouts of the tile kernels' bounded waits since the last call (the
// kernels leave such a tile unfiltered and count it): 0 when none.
int pass2_wait_timeouts(uint32_t *count);
// Packed 16x2 form; requires bit_depth <= 14, 4:2:0 or 4:0:0, coefficients in [-128, 127].
int launch_pass2_packed(cudaStream_t st, const Pass2Args &a, bool do_sao, bool do_alf, uint64_t *launches);

// ---------------------------------------------------------------- recon-side LMCS, output dump (recon.cu)
struct RectPiece {  // a piece of a forward-map rectangle, inside the plane, on whole coverage cells
  uint32_t x, y, w, h;
};
// How many of a call's rectangles cover each cell of a grid of 2^sh x 2^sh
// luma samples (every rectangle edge of the call lies on the grid), and the
// box the rectangles span.
struct FwdCover {
  uint32_t *cnt;       // pitch x ceil(height / 2^sh) counters: zero before the count launch, zero again after the apply launch
  uint32_t pitch, sh;  // counters per row, grid shift
  uint32_t x0, y0, x1, y1;
};
struct ResPiece {  // a piece of a chroma TB's residual add: <= 1024 samples
  uint32_t x, y, w, h;
  uint32_t plane, var_scale;
  uint64_t res_offset;  // residual of (x, y)
  uint32_t res_pitch, pad;
};
struct CvsTables {
  uint32_t pivot[17], chroma_scale[16];
  uint32_t mn, mx, bd;
};
struct OutPlanes {
  DPlane p[3];
  uint32_t x0[3], y0[3], w[3];
  uint64_t n[3], total;  // output samples per plane, and in all
};
int launch_lmcs_fwd_lut(cudaStream_t st, uint16_t *d_lut, const h266_lmcs_derived &l, uint64_t *launches);
// The forward map of a rectangle list in two launches: the coverage count of
// every cell (one warp per piece), then one pass over the span box mapping
// each sample as many times as rectangles cover it.
int launch_lmcs_fwd_cover(cudaStream_t st, DPlane p, const uint16_t *d_lut, const RectPiece *d_pieces, uint32_t n,
                          const FwdCover &c, bool check, uint32_t *d_err, uint64_t *launches);
// The chroma TBs of a residual-add call on a grid of 2^sh x 2^sh chroma
// samples (every TB edge of the call lies on it): per plane the owner of
// each cell (TB index + 1, 0 none) and the box the plane's TBs span.
struct ResCover {
  uint32_t *own[2];  // Cb, Cr: pitch x ceil(height / 2^sh) owners, all 0 between calls
  uint32_t pitch[2], sh;
  uint32_t x0[2], y0[2], x1[2], y1[2];
};
// The residual add in two launches when the call's TBs are pairwise
// disjoint: the owner of every cell (one warp per TB; a cell claimed twice
// raises *overlap), then one pass over each plane's box adding each
// sample's residual; with *overlap raised the pass returns at once, leaving
// the planes as they were (and the owners set) for the ordered launches of
// launch_chroma_residual.
int launch_chroma_residual_cover(cudaStream_t st, DPlane cb, DPlane cr, const h266_chroma_res_block *d_blocks,
                                 uint32_t n, const int32_t *d_res, int bd, const ResCover &c, uint32_t *d_overlap,
                                 uint64_t *launches);
int launch_lmcs_cvs(cudaStream_t st, DPlane luma, const h266_lmcs_cvs_block *d_blocks, uint32_t n, int size_y,
                    const CvsTables &t, uint32_t *d_out, uint64_t *launches);
int launch_chroma_residual(cudaStream_t st, DPlane cb, DPlane cr, const ResPiece *d_pieces, uint32_t n,
                           const int32_t *d_res, int bd, uint64_t *launches);
int launch_output_dump(cudaStream_t st, const OutPlanes &o, uint8_t *d_dst, bool wide, uint64_t *launches);

// Encoder chroma ALF / CC-ALF trials (alf_enc.cu): per-CTB chroma SSE of a
// against b into d_sse[ctb * cols + col]; then the first-minimum pick per CTB
// and the copy of the chosen trial plane's CTB region into dst.
int launch_ctb_sse(cudaStream_t st, DPlane a, DPlane b, int cw, int ch, int w_ctbs, int n, unsigned long long *d_sse,
                   int cols, int col, uint64_t *launches);
int launch_trial_pick_commit(cudaStream_t st, const unsigned long long *d_sse, int cols, int n, int8_t *d_pick,
                             DPlane dst, const uint16_t *d_trials, int64_t trial_samples, int trial_pitch, int cw,
                             int ch, int w_ctbs, uint64_t *launches);

// Encoder SAO decision (sao_enc.cu): statistics per (CTB, component) into
// d_stats (sao_stats_bytes), then the per-CTB decision into d_out.
size_t sao_stats_bytes(int n_ctbs);
// Chroma SAO merge (sao_enc.cu): one launch per CTB anti-diagonal; d_merged
// is written CTB by CTB (each launch reads the previous diagonal's records).
int launch_sao_chroma_merge(cudaStream_t st, const DPlane src[2], const DPlane pre[2], int bd, int chr_ctb,
                            int w_ctbs, int h_ctbs, const h266_sao_ctb_params *d_indep, h266_sao_ctb_params *d_merged,
                            uint8_t *d_map, void *d_work, uint64_t *launches);
inline size_t sao_merge_work_bytes(size_t n_ctbs) { return n_ctbs * 3 * 8 + n_ctbs * 4; }
// Batched merge: one launch per anti-diagonal over many pictures.
// fill_sao_merge_args writes one picture's parameters (sao_merge_args_size()
// bytes; d_work laid out as sao_merge_work_bytes, its per-CTB counts zeroed by
// the caller); d_first holds per diagonal the n + 1 prefix sums of the
// pictures' CTB counts on it, h_totals the diagonals' totals.
size_t sao_merge_args_size();
void fill_sao_merge_args(void *out, const DPlane src[2], const DPlane pre[2], int bd, int chr_ctb, int w_ctbs,
                         int h_ctbs, const h266_sao_ctb_params *d_indep, h266_sao_ctb_params *d_merged, uint8_t *d_map,
                         void *d_work);
int launch_sao_chroma_merge_batch(cudaStream_t st, const void *d_args, const uint32_t *d_first, int n, int n_diags,
                                  const uint32_t *h_totals, uint64_t *launches);
int launch_sao_decide(cudaStream_t st, const DPlane src[3], const DPlane rec[3], int bd, int log2, int w_ctbs,
                      int h_ctbs, bool luma_on, bool chroma_on, void *d_stats, uint32_t *d_err,
                      h266_sao_ctb_params *d_out, uint64_t *launches);

// Encoder luma ALF trials (packed form): `trials` filter-set slots of
// a.tables.luma_packed evaluated on the pre-ALF luma a.src[0] against the
// original `orig`; d_sse[ctb * cols + 0] += pre-ALF SSE, [.. + 1 + t] += SSE
// of trial t (d_sse zeroed by the caller).  Then per CTB the decision, written
// into d_ctbs[].luma_set (slot or -1) and d_decision[].
constexpr int kAlfMaxTrials = 17;
int launch_alf_luma_trials(cudaStream_t st, const Pass2Args &a, const DPlane &orig, int trials, int cols,
                           unsigned long long *d_sse, uint64_t *launches);
int launch_alf_luma_decide(cudaStream_t st, CtbDev *d_ctbs, int n, unsigned long long *d_sse, int cols, int trials_run,
                           int16_t *d_decision, uint64_t *launches);
int pass2_packed_variant(Pass2Args &a, bool do_sao, bool do_alf, uint32_t *ctas);
// Batched packed pass: fills a's tile grid (a.tile_h chooses the tile height
// for CTBs of 64 and 128), returns the kernel variant (0..11) and the
// picture's CTA count; pictures of one variant share a launch.  With
// ctas_per_sm > 0 the launch is persistent: that many CTAs per SM drain the
// variant's (picture, tile) items through the counter *d_queue (zero at launch).
constexpr int kPass2Variants = 12;
int launch_pass2_packed_batch(cudaStream_t st, int variant, const Pass2Args *d_args, const uint32_t *d_first, int n,
                              uint32_t ctas, int ctas_per_sm, uint32_t *d_queue, uint64_t *launches);

}  // namespace h266
