// Deblocking (H.266 §8.8.3) for the B200 filter chain.
//
// Host side: the reference walks its CU list in decode order and filters every
// edge segment in place, sequentially (src/deblock.rs:687-983).  The walk's
// edge derivation -- positions, bS, maxFilterLength, beta / tC -- reads no
// samples, so it is done up front here and produces an explicit segment list.
// Segments are then grouped into components: two segments of the same pass
// and plane that lie on the same 4-line (luma) or 2-line (chroma) band and
// whose sample footprints overlap along the edge normal are in one component.
// A segment's footprint is [pos - R(mflP), pos + R(mflQ)) with R(m) = 4 for
// m <= 3 and m + 1 otherwise: every sample the decision or the filters of
// src/deblock.rs:1224-2075 read or write lies inside it.  Segments of
// different components therefore touch disjoint samples and commute; inside
// a component the segments keep the reference's processing order.  The
// vertical pass runs to completion before the horizontal one, as in
// apply_deblocking_clipped (src/deblock.rs:540-615).
//
// Device side: one thread per component replays its segments with the
// reference's clamped reads and bounds-checked Clip1 writes on global memory.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <numeric>

#include "internal.h"
#include "tma.cuh"

namespace h266 {
namespace {

// The edge derivation below runs on the host (the general plan) and on the
// device (the side-information builder for pictures without chained edges):
// the same functions, compiled for both.
#define H266_HD __host__ __device__

// ---------------------------------------------------------------- tables
// Table 43 (β′, tC′) as in src/deblock.rs:401-418.
#define H266_BETA_TABLE \
  0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 6, 7, 8, 9, 10, 11,  \
  12, 13, 14, 15, 16, 17, 18, 20, 22, 24, 26, 28, 30, 32, 34, 36, 38, 40, 42, 44, 46, 48,  \
  50, 52, 54, 56, 58, 60, 62, 64, 66, 68, 70, 72, 74, 76, 78, 80, 82, 84, 86, 88
#define H266_TC_TABLE \
  0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 3, 4, 4, 4,  \
  4, 5, 5, 5, 5, 7, 7, 8, 9, 10, 10, 11, 13, 14, 15, 17, 19, 21, 24, 25, 29, 33,  \
  36, 41, 45, 51, 57, 64, 71, 80, 89, 100, 112, 125, 141, 157, 177, 198, 222, 250, 280, 314, 352, 395
#ifndef __CUDA_ARCH__
const int kBeta[64] = {H266_BETA_TABLE};
const int kTc[66] = {H266_TC_TABLE};
#endif
__constant__ int kBetaDev[64] = {H266_BETA_TABLE};  // the same tables for device code
__constant__ int kTcDev[66] = {H266_TC_TABLE};

H266_HD inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// eqs. 1276-1279 (src/deblock.rs:424-452)
H266_HD inline int beta_of(int q, int bd) {
#ifdef __CUDA_ARCH__
  return kBetaDev[clampi(q, 0, 63)] * (1 << (bd - 8));
#else
  return kBeta[clampi(q, 0, 63)] * (1 << (bd - 8));
#endif
}
H266_HD inline int tc_of(int q, int bd) {
#ifdef __CUDA_ARCH__
  int t = kTcDev[clampi(q, 0, 65)];
#else
  int t = kTc[clampi(q, 0, 65)];
#endif
  if (bd < 10) return (t + (1 << (9 - bd))) >> (10 - bd);
  return t * (1 << (bd - 10));
}

// ---------------------------------------------------------------- CU geometry
// The per-CU transform-block queries of src/deblock.rs:163-320, for one CU.
struct Cu {
  const h266_deblock_cu &c;
  H266_HD uint32_t rel(int lx, int ly, bool vert) const {
    return vert ? (uint32_t)clampi(lx - (int)c.x, 0, (int)c.w - 1) : (uint32_t)clampi(ly - (int)c.y, 0, (int)c.h - 1);
  }
  H266_HD int split_index(uint32_t r) const {
    int idx = 0;
    for (int i = 0; i < c.tb_split.n_bounds; ++i)
      if (r >= c.tb_split.bounds[i]) idx = i + 1;
    return idx;
  }
  H266_HD uint32_t split_len(uint32_t r, uint32_t dim) const {
    uint32_t lo = 0, hi = dim;
    for (int i = 0; i < c.tb_split.n_bounds; ++i) {
      if (r < c.tb_split.bounds[i]) {
        hi = c.tb_split.bounds[i];
        break;
      }
      lo = c.tb_split.bounds[i];
    }
    return hi - lo;
  }
  H266_HD bool coded(uint32_t comp, int lx, int ly) const {  // tu_coded_at
    if (c.has_tu64) {
      uint32_t tx = std::min(rel(lx, ly, true) / 64, 1u), ty = std::min(rel(lx, ly, false) / 64, 1u);
      return comp == 0 ? c.tu64.y[ty][tx] : (comp == 1 ? c.tu64.cb[ty][tx] : c.tu64.cr[ty][tx]);
    }
    if (c.has_tb_split && (comp == 0 || !c.tb_split.luma_only)) {
      int i = split_index(rel(lx, ly, c.tb_split.vertical != 0));
      return comp == 0 ? c.tb_split.y_coded[i] : (comp == 1 ? c.tb_split.cb_coded[i] : c.tb_split.cr_coded[i]);
    }
    return comp == 0 ? c.tu_y_coded : (comp == 1 ? c.tu_cb_coded : c.tu_cr_coded);
  }
  H266_HD uint32_t tb_len(int lx, int ly, bool vert, bool chroma) const {  // luma_tb_len / chroma_tb_len (luma units)
    uint32_t dim = vert ? c.w : c.h;
    if (c.has_tu64 && dim > 64) return std::min(dim - (rel(lx, ly, vert) / 64) * 64, 64u);
    if (c.has_tb_split && (c.tb_split.vertical != 0) == vert && !(chroma && c.tb_split.luma_only))
      return split_len(rel(lx, ly, vert), dim);
    return dim;
  }
  H266_HD bool tb_boundary(uint32_t off, bool vert, bool chroma) const {  // is_{luma,chroma}_tb_boundary
    uint32_t dim = vert ? c.w : c.h;
    if (off == 0 || off >= dim) return false;
    if (c.has_tu64 && dim > 64) return off % 64 == 0;
    if (c.has_tb_split && (c.tb_split.vertical != 0) == vert && !(chroma && c.tb_split.luma_only)) {
      for (int i = 0; i < c.tb_split.n_bounds; ++i)
        if (c.tb_split.bounds[i] == off) return true;
    }
    return false;
  }
};

#ifndef __CUDA_ARCH__
const h266_deblock_mv_cell kNoMotion = {};  // DeblockMvCell::default()
#endif
__device__ const h266_deblock_mv_cell kNoMotionDev = {};

struct MvGrid {  // `g` points to a grid descriptor whose cells are reachable by the caller's side
  const h266_deblock_mv_grid *g;
  H266_HD const h266_deblock_mv_cell &at(int x, int y) const {  // DeblockMvGrid::at_luma
#ifdef __CUDA_ARCH__
    const h266_deblock_mv_cell &none = kNoMotionDev;
#else
    const h266_deblock_mv_cell &none = kNoMotion;
#endif
    if (!g || x < 0 || y < 0) return none;
    uint64_t cx = (uint64_t)x / 4, cy = (uint64_t)y / 4;
    if (cx >= g->cells_w || cy >= g->cells_h) return none;
    return g->cells[cy * g->cells_w + cx];
  }
};

H266_HD inline bool mv_far(const int32_t *a, const int32_t *b) { return abs(a[0] - b[0]) >= 8 || abs(a[1] - b[1]) >= 8; }

// §8.8.3.5 motion arm, src/deblock.rs:992-1045
H266_HD inline bool motion_differs(const h266_deblock_mv_cell &p, const h266_deblock_mv_cell &q) {
  int np = (p.pred_l0 != 0) + (p.pred_l1 != 0), nq = (q.pred_l0 != 0) + (q.pred_l1 != 0);
  if (np != nq) return true;
  if (np == 0) return false;
  if (np == 1) {
    int pp = p.pred_l0 ? p.poc_l0 : p.poc_l1, qp = q.pred_l0 ? q.poc_l0 : q.poc_l1;
    if (pp != qp) return true;
    return mv_far(p.pred_l0 ? p.mv_l0 : p.mv_l1, q.pred_l0 ? q.mv_l0 : q.mv_l1);
  }
  bool straight_refs = p.poc_l0 == q.poc_l0 && p.poc_l1 == q.poc_l1;
  bool swapped_refs = p.poc_l0 == q.poc_l1 && p.poc_l1 == q.poc_l0;
  if (!straight_refs && !swapped_refs) return true;
  bool straight = mv_far(p.mv_l0, q.mv_l0) || mv_far(p.mv_l1, q.mv_l1);
  bool crossed = mv_far(p.mv_l0, q.mv_l1) || mv_far(p.mv_l1, q.mv_l0);
  if (p.poc_l0 != p.poc_l1) return straight_refs ? straight : crossed;
  return straight && crossed;
}

struct PlaneCfg {
  uint32_t comp, sub_w, sub_h;
  int beta_off, tc_off, qp_off, bd;
  uint32_t ctb;
};

struct Emitted {  // a segment in emission (reference) order: its index in the list
  EdgeSeg s;
};

class Walker {
 public:
  // `grid` is caller-owned storage for the 4x4 cell -> CU map, reused across
  // calls so that no call allocates it anew.
  Walker(const h266_deblock_cu *cus, size_t n, int pw, int ph, std::vector<int32_t> &grid)
      : cus_(cus), n_(n), grid_(grid) {
    cw_ = (pw + 3) / 4;
    ch_ = (ph + 3) / 4;
    grid_.assign((size_t)cw_ * ch_, -1);
    for (size_t i = 0; i < n; ++i) {  // CuGrid::build, later CUs win
      const h266_deblock_cu &c = cus[i];
      int x0 = c.x / 4, y0 = c.y / 4;
      int x1 = std::min<int64_t>(((int64_t)c.x + c.w + 3) / 4, cw_), y1 = std::min<int64_t>(((int64_t)c.y + c.h + 3) / 4, ch_);
      for (int y = y0; y < y1; ++y)
        for (int x = x0; x < x1; ++x) grid_[(size_t)y * cw_ + x] = (int32_t)i;
    }
  }
  int64_t at(int x, int y) const {
    if (x < 0 || y < 0 || x / 4 >= cw_ || y / 4 >= ch_) return -1;
    return grid_[(size_t)(y / 4) * cw_ + x / 4];
  }
  // deblock_cu_dir (src/deblock.rs:707-983) for every CU, recording segments.
  void walk(const PlaneCfg &pc, bool vert, const MvGrid &mv, const uint32_t *nf, uint64_t n_nf,
            std::vector<Emitted> &out) const;

 private:
  const h266_deblock_cu *cus_;
  size_t n_;
  int cw_, ch_;
  std::vector<int32_t> &grid_;
};

// `mv`: the motion lookup (MvGrid, or per-CU motion on the device); mv.g
// non-null when the picture has a motion grid.
#pragma nv_exec_check_disable
template <class Mv>
H266_HD inline int bs_of(uint32_t comp, const h266_deblock_cu &p, const h266_deblock_cu &q, const Mv &mv, int px,
                         int py, int qx, int qy, bool is_tb, bool idc2) {  // derive_bs, src/deblock.rs:1055-1119
  if (comp == 0 ? (p.bdpcm_luma && q.bdpcm_luma) : (p.bdpcm_chroma && q.bdpcm_chroma)) return 0;
  if (p.intra || q.intra || p.ciip || q.ciip) return 2;
  if (is_tb && (Cu{p}.coded(comp, px, py) || Cu{q}.coded(comp, qx, qy))) return 1;
  if (comp != 0 || !idc2) return 0;
  if ((p.ibc != 0) != (q.ibc != 0)) return 1;
  if (p.ibc) {
    if (mv.g) return mv_far(mv.at(px, py).mv_l0, mv.at(qx, qy).mv_l0) ? 1 : 0;
    return 0;
  }
  if (mv.g && motion_differs(mv.at(px, py), mv.at(qx, qy))) return 1;
  return 0;
}

// The walk geometry of a CU for one (plane, pass), shared by its edges
// (deblock_cu_dir, src/deblock.rs:707-760).
struct CuWalkGeo {
  uint32_t n_cb, n_other, step, seg, nsb, sb, n8, last_sb, ctb_h_c;
  bool chroma, filter_edge, off_grid;  // off_grid: a chroma CU off the 8-sample chroma edge grid
};

H266_HD inline CuWalkGeo cu_walk_geo(const h266_deblock_cu &cu, const PlaneCfg &pc, bool vert, const uint32_t *nf,
                                     uint64_t n_nf) {
  CuWalkGeo g;
  g.chroma = pc.comp != 0;
  g.off_grid = g.chroma && ((vert ? cu.x / pc.sub_w : cu.y / pc.sub_h) % 8) != 0;
  g.n_cb = vert ? cu.w : cu.h;
  g.n_other = vert ? cu.h : cu.w;
  const uint32_t lead = vert ? cu.x : cu.y;
  bool gated = false;
  for (uint64_t i = 0; i < n_nf; ++i) gated |= nf[i] == lead;
  g.filter_edge = lead != 0 && !gated;
  g.step = g.chroma ? 8 * (vert ? pc.sub_w : pc.sub_h) : 4;
  g.seg = g.chroma ? 2 * (vert ? pc.sub_h : pc.sub_w) : 4;
  g.nsb = 1;
  if (!g.chroma && cu.has_num_sb) g.nsb = std::max(vert ? cu.num_sb_x : cu.num_sb_y, 1u);
  g.sb = std::max(8u, g.n_cb / g.nsb);
  g.n8 = std::max(g.n_cb / 8, 1u);
  g.last_sb = std::min(g.n8 - 1, g.nsb - 1);
  g.ctb_h_c = pc.ctb / std::max(pc.sub_h, 1u);
  return g;
}

// Along one edge only the P-side CU and the bS inputs change; the
// maxFilterLengths, qP and flags that depend on the P-side CU are kept while
// it stays the same (a fresh WalkMemo recomputes them: same values).
struct WalkMemo {
  int64_t pi = -2;
  uint32_t mp = 0, mq = 0;
  int qp = 0;
};

// The segment at position k along the edge at offset `off` of CU `idx`
// (deblock_cu_dir's inner loop, src/deblock.rs:760-983): emitted when it
// filters anything.  `grid.at(x, y)` is the CU covering luma sample (x, y)
// (CuGrid::cu_at), -1 for none.
#pragma nv_exec_check_disable
template <class Grid, class Mv, class Emit>
H266_HD inline void walk_segment(const h266_deblock_cu *cus_, const Grid &grid, const PlaneCfg &pc, bool vert,
                                 const Mv &mv, size_t idx, const CuWalkGeo &g, uint32_t off, bool is_tb, bool is_sb,
                                 uint32_t k, Emit &emit, WalkMemo &memo) {
  const h266_deblock_cu &cu = cus_[idx];
  const bool chroma = g.chroma, filter_edge = g.filter_edge;
  const uint32_t n_cb = g.n_cb, nsb = g.nsb, sb = g.sb, n8 = g.n8, ctb_h_c = g.ctb_h_c;
  Cu q_geo{cu};
    const int qx = (int)(vert ? cu.x + off : cu.x + k), qy = (int)(vert ? cu.y + k : cu.y + off);
    const int px = vert ? qx - 1 : qx, py = vert ? qy : qy - 1;
    int64_t pi = off == 0 ? grid.at(px, py) : (int64_t)idx;
    if (pi < 0 || (off == 0 && pi == (int64_t)idx)) return;
    const h266_deblock_cu &p = cus_[pi];
    const int bs = bs_of(pc.comp, p, cu, mv, px, py, qx, qy, is_tb, is_sb);
    if (bs == 0) return;
    uint32_t mp, mq;
    int qp;
    const bool ctb_row = !chroma && !vert && off == 0 && pc.ctb > 0 && cu.y % pc.ctb == 0;
    if (pi == memo.pi) {
      mp = memo.mp;
      mq = memo.mq;
      qp = memo.qp;
    } else if (!chroma) {
      mp = mq = 0;
      if (is_tb) {
        uint32_t wq = q_geo.tb_len(qx, qy, vert, false), wp = Cu{p}.tb_len(px, py, vert, false);
        if (wp <= 4 || wq <= 4) mp = mq = 1;
        else {
          mp = wp >= 32 ? 7 : 3;
          mq = wq >= 32 ? 7 : 3;
        }
      }
      if (is_sb) {  // §8.8.3.4 overlay, src/deblock.rs:856-901
        if (off == 0) {
          if (nsb > 1) mq = std::min(mq, 5u);
          if (p.has_num_sb) mp = std::min(mp, 5u);
        } else {
          auto tb_at = [&](int64_t z) {
            if (z < 0 || z >= (int64_t)n_cb) return false;
            return z == 0 ? filter_edge : q_geo.tb_boundary((uint32_t)z, vert, false);
          };
          if (is_tb) {
            mp = std::min(mp, 5u);
            mq = std::min(mq, 5u);
          } else if (tb_at((int64_t)off - 4) || tb_at((int64_t)off + 4)) {
            mp = mq = 1;
          } else if (off / sb == 1 || off / sb == n8 - 1 || tb_at((int64_t)off - sb) || tb_at((int64_t)off + sb)) {
            mp = mq = 2;
          } else {
            mp = mq = 3;
          }
        }
      }
      qp = (p.qp_y + cu.qp_y + 1) >> 1;  // eq. 1274 (no LADF)
    } else {
      const uint32_t sub = vert ? pc.sub_w : pc.sub_h;
      const uint32_t wq = q_geo.tb_len(qx, qy, vert, true) / sub, wp = Cu{p}.tb_len(px, py, vert, true) / sub;
      if (wp >= 8 && wq >= 8) {
        const bool row = !vert && off == 0 && ctb_h_c > 0 && (cu.y / pc.sub_h) % ctb_h_c == 0;
        mp = row ? 1 : 3;
        mq = 3;
      } else {
        mp = mq = 1;
      }
      auto pick = [&](const h266_deblock_cu &c) {  // src/deblock.rs:1155-1163
        if (c.qp_c[0] == INT32_MIN) return clampi(c.qp_y + pc.qp_off, 0, 63);
        if (c.joint_cbcr2) return (int)c.qp_c[2];
        return (int)c.qp_c[pc.comp == 1 ? 0 : 1];
      };
      qp = (pick(p) + pick(cu) + 1) >> 1;  // eq. 1343
    }
    memo.pi = pi;
    memo.mp = mp;
    memo.mq = mq;
    memo.qp = qp;
    const int beta = beta_of(qp + pc.beta_off * 2, pc.bd);
    const int tc = tc_of(qp + 2 * (bs - 1) + pc.tc_off * 2, pc.bd);
    if (tc == 0) return;  // every filter arm is a no-op at tC = 0
    if (chroma && mp == 1 && mq == 1 && bs != 2) return;  // src/deblock.rs:1823, 1888
    Emitted e;
    e.s.x = (uint16_t)(chroma ? qx / (int)pc.sub_w : qx);
    e.s.y = (uint16_t)(chroma ? qy / (int)pc.sub_h : qy);
    e.s.beta = (uint16_t)beta;
    e.s.tc = (uint16_t)tc;
    e.s.plane = (uint8_t)pc.comp;
    e.s.bs = (uint8_t)bs;
    e.s.mfl = (uint8_t)(mp << 4 | mq);
    e.s.flags = (uint8_t)((vert ? 1 : 0) | (ctb_row ? 2 : 0) | (p.plt ? 4 : 0) | (cu.plt ? 8 : 0));
    emit(e.s);
}

// deblock_cu_dir (src/deblock.rs:707-983) for CU `idx`: every edge segment it
// owns, in the reference's order, passed to `emit`.
#pragma nv_exec_check_disable
// `only_off` >= 0 restricts the walk to the edge at that offset inside the CU
// (the device runs one thread per offset).
template <class Grid, class Mv, class Emit>
H266_HD void walk_cu(const h266_deblock_cu *cus_, const Grid &grid, const PlaneCfg &pc, bool vert, const Mv &mv,
                     const uint32_t *nf, uint64_t n_nf, size_t idx, Emit &emit, int only_off = -1) {
  const h266_deblock_cu &cu = cus_[idx];
  const CuWalkGeo g = cu_walk_geo(cu, pc, vert, nf, n_nf);
  if (g.off_grid) return;
  Cu q_geo{cu};
  for (uint32_t off = only_off >= 0 ? (uint32_t)only_off : 0; off < g.n_cb; off += g.step) {
    if (only_off >= 0 && off != (uint32_t)only_off) break;
    const bool is_tb = off == 0 ? g.filter_edge : q_geo.tb_boundary(off, vert, g.chroma);
    const bool is_sb = !g.chroma && off % g.sb == 0 && off / g.sb <= g.last_sb && (off > 0 || g.filter_edge);
    if (!is_tb && !is_sb) continue;
    WalkMemo memo;
    for (uint32_t k = 0; k < g.n_other; k += g.seg)
      walk_segment(cus_, grid, pc, vert, mv, idx, g, off, is_tb, is_sb, k, emit, memo);
  }
}

struct VectorEmit {  // host: the segment list in emission order
  std::vector<Emitted> &out;
  void operator()(const EdgeSeg &s) { out.push_back(Emitted{s}); }
};

void Walker::walk(const PlaneCfg &pc, bool vert, const MvGrid &mv, const uint32_t *nf, uint64_t n_nf,
                  std::vector<Emitted> &out) const {
  VectorEmit emit{out};
  for (size_t idx = 0; idx < n_; ++idx) walk_cu(cus_, *this, pc, vert, mv, nf, n_nf, idx, emit);
}

inline int reach(int m) { return m <= 3 ? 4 : m + 1; }
__device__ __forceinline__ int reach_d(int m) { return m <= 3 ? 4 : m + 1; }

// Groups one (pass, plane) segment list into components and appends them.
// Components come out band by band, by footprint start inside a band, with
// their members in emission (reference) order.  Segments are bucketed by band
// in emission order; decode order visits the CUs crossing a band from its low
// end to its high end (z-scan inside a CTB, raster / tile order between CTBs),
// so a bucket is normally sorted by footprint start already and the pass is
// linear.  A bucket that is not (CU lists in an unusual order) is sorted, and
// its components' members are put back in emission order.
struct GroupScratch {
  struct Item {  // a segment with its footprint and emission index, bucketed by band
    EdgeSeg s;
    int32_t start, end;
    uint32_t i;
  };
  std::vector<uint32_t> head;
  std::vector<Item> items, members;
};

void group(const std::vector<Emitted> &segs, std::vector<EdgeSeg> &dst, std::vector<uint32_t> &comp,
           uint32_t &max_len, GroupScratch &g) {
  const size_t n = segs.size();
  if (n == 0) return;
  uint32_t max_band = 0;
  for (size_t i = 0; i < n; ++i) {
    const EdgeSeg &s = segs[i].s;
    max_band = std::max<uint32_t>(max_band, (s.flags & 1) ? s.y : s.x);
  }
  g.head.assign((size_t)max_band + 2, 0);
  for (size_t i = 0; i < n; ++i) {
    const EdgeSeg &s = segs[i].s;
    ++g.head[(size_t)((s.flags & 1) ? s.y : s.x) + 1];
  }
  for (size_t b = 1; b < g.head.size(); ++b) g.head[b] += g.head[b - 1];
  g.items.resize(n);
  {
    std::vector<uint32_t> &cur = g.head;  // used as the fill cursor, restored below
    for (size_t i = 0; i < n; ++i) {
      const EdgeSeg &s = segs[i].s;
      const bool vert = s.flags & 1;
      const int pos = vert ? s.x : s.y;
      g.items[cur[vert ? s.y : s.x]++] =
          GroupScratch::Item{s, pos - reach(s.mfl >> 4), pos + reach(s.mfl & 15), (uint32_t)i};
    }
    for (size_t b = g.head.size() - 1; b > 0; --b) g.head[b] = g.head[b - 1];  // cursor[b] ended at start[b + 1]
    g.head[0] = 0;
  }
  const size_t d0 = dst.size();
  dst.resize(d0 + n);
  EdgeSeg *out = dst.data() + d0;
  size_t o = 0;
  uint32_t longest = max_len;
  auto by_start = [](const GroupScratch::Item &a, const GroupScratch::Item &b) { return a.start < b.start; };
  for (size_t b = 0; b + 1 < g.head.size(); ++b) {
    GroupScratch::Item *lo = g.items.data() + g.head[b], *hi = g.items.data() + g.head[b + 1];
    if (lo == hi) continue;
    const bool sorted = std::is_sorted(lo, hi, by_start);
    if (!sorted) std::stable_sort(lo, hi, by_start);  // ties keep emission order
    for (GroupScratch::Item *i = lo; i < hi;) {
      GroupScratch::Item *j = i + 1;
      int32_t e = i->end;
      while (j < hi && j->start < e) {
        e = std::max(e, j->end);
        ++j;
      }
      comp.push_back((uint32_t)(d0 + o));
      if (sorted || j - i == 1) {
        for (GroupScratch::Item *t = i; t < j; ++t) out[o++] = t->s;
      } else {
        g.members.assign(i, j);
        std::sort(g.members.begin(), g.members.end(),
                  [](const GroupScratch::Item &a, const GroupScratch::Item &b) { return a.i < b.i; });
        for (const GroupScratch::Item &m : g.members) out[o++] = m.s;
      }
      longest = std::max<uint32_t>(longest, (uint32_t)(j - i));
      i = j;
    }
  }
  max_len = longest;
}

// Fills the band index of both passes from the component lists.
void index_bands(const h266_picture &pic, DeblockPlan &plan) {
  const h266_plane *pl[3] = {&pic.luma, &pic.cb, &pic.cr};
  for (int d = 0; d < 2; ++d) {
    std::vector<uint32_t> &bf = plan.band_first[d];
    bf.clear();
    const std::vector<uint32_t> &comp = plan.comp[d];
    const std::vector<EdgeSeg> &segs = plan.segs[d];
    const uint32_t n_comp = (uint32_t)comp.size() - 1;
    uint32_t c = 0;
    for (int p = 0; p < 3; ++p) {
      const uint32_t unit = p ? 2 : 4;
      const uint32_t dim = d == 0 ? pl[p]->height : pl[p]->width;
      const uint32_t nb = (uint64_t)pl[p]->width * pl[p]->height ? (dim + unit - 1) / unit : 0;
      plan.band_off[d][p] = (uint32_t)bf.size();
      plan.n_bands[d][p] = nb;
      // components of plane p are contiguous, sorted by band coordinate
      for (uint32_t b = 0; b <= nb; ++b) {
        while (c < n_comp && segs[comp[c]].plane == p && (d == 0 ? segs[comp[c]].y : segs[comp[c]].x) / unit < b) ++c;
        bf.push_back(c);
      }
      while (c < n_comp && segs[comp[c]].plane == p) ++c;  // bands beyond the plane
    }
  }
}

// Fills the component ranges of the tile kernel.  A vertical-pass component
// runs in every tile whose columns its footprint reaches and whose rows
// widened by the halo hold its band (the horizontal pass of those rows reads
// its output); a horizontal-pass component runs in the tile holding its band
// whose rows its footprint reaches.  Footprints are clipped to the plane, so
// components touching no sample of it are in no range.
void index_tiles(const h266_picture &pic, uint32_t cfi, DeblockPlan &plan) {
  plan.tiles_ok = false;
  const int T = kDeblockTile;
  const int w = (int)pic.luma.width, h = (int)pic.luma.height;
  plan.tiles_x = (uint32_t)((w + T - 1) / T);
  plan.tiles_y = (uint32_t)((h + T - 1) / T);
  const bool chroma = (uint64_t)pic.cb.width * pic.cb.height != 0 || (uint64_t)pic.cr.width * pic.cr.height != 0;
  if (cfi > 1 || (cfi == 0 && chroma)) return;
  if (chroma && (pic.cb.width != (pic.luma.width + 1) / 2 || pic.cb.height != (pic.luma.height + 1) / 2 ||
                 pic.cr.width != pic.cb.width || pic.cr.height != pic.cb.height))
    return;
  const int tiles_x = (int)plan.tiles_x, tiles_y = (int)plan.tiles_y;
  std::vector<uint32_t> &tb = plan.tile_bounds;
  tb.clear();
  // per tile and pass: staged segments per plane, checked against the shared lists
  thread_local std::vector<uint32_t> load;
  load.assign((size_t)tiles_x * tiles_y * 3, 0);
  for (int d = 0; d < 2; ++d) {
    std::fill(load.begin(), load.end(), 0);
    const std::vector<uint32_t> &comp = plan.comp[d];
    const std::vector<EdgeSeg> &segs = plan.segs[d];
    for (int p = 0; p < 3; ++p) {
      plan.tb_off[d][p] = (uint32_t)tb.size();
      const uint32_t nb = plan.n_bands[d][p];
      if (!nb) continue;
      const int tp = p ? T / 2 : T, halo = p ? kDeblockHaloC : kDeblockHaloY, unit = p ? 2 : 4;
      const int along = d == 0 ? (p ? (int)pic.cb.width : w) : (p ? (int)pic.cb.height : h);
      const int n_t = d == 0 ? tiles_x : tiles_y;  // tiles along the footprint axis
      const uint32_t *bf = plan.band_first[d].data() + plan.band_off[d][p];
      const size_t base = tb.size();
      tb.resize(base + (size_t)nb * n_t * 2);
      thread_local std::vector<int32_t> fs, fe;  // clipped footprints of one band's components
      for (uint32_t b = 0; b < nb; ++b) {
        const uint32_t c0 = bf[b], c1 = bf[b + 1];
        fs.resize(c1 - c0);
        fe.resize(c1 - c0);
        for (uint32_t c = c0; c < c1; ++c) {
          const EdgeSeg &f = segs[comp[c]];
          const int pos = (f.flags & 1) ? f.x : f.y;
          int s = pos - reach(f.mfl >> 4), e = pos + reach(f.mfl & 15);
          for (uint32_t i = comp[c] + 1; i < comp[c + 1]; ++i) {
            const EdgeSeg &g = segs[i];
            const int q = (g.flags & 1) ? g.x : g.y;
            s = std::min(s, q - reach(g.mfl >> 4));
            e = std::max(e, q + reach(g.mfl & 15));
          }
          if (e - s > halo) return;  // longer than the halo: strip kernels
          fs[c - c0] = std::max(s, 0);
          fe[c - c0] = std::min(e, along);
        }
        uint32_t lo = c0, hi = c0;
        for (int t = 0; t < n_t; ++t) {
          const int t0 = t * tp, t1 = std::min((t + 1) * tp, along);
          while (lo < c1 && fe[lo - c0] <= t0) ++lo;
          if (hi < lo) hi = lo;
          while (hi < c1 && fs[hi - c0] < t1) ++hi;
          tb[base + ((size_t)b * n_t + t) * 2] = lo;
          tb[base + ((size_t)b * n_t + t) * 2 + 1] = hi;
          // count the segments of the tiles that take this band's range (the
          // tile kernel stages them in shared lists of kTileListY / kTileListC)
          const uint32_t n = comp[hi] - comp[lo];
          if (!n) continue;
          if (d == 0) {
            const int band = (int)b * unit;
            const int ty0 = band - halo < 0 ? 0 : (band - halo) / tp;
            const int ty1 = std::min(tiles_y - 1, (band + unit + halo - 1) / tp);
            for (int ty = ty0; ty <= ty1; ++ty) load[((size_t)ty * tiles_x + t) * 3 + p] += n;
          } else {
            const int tx = (int)b * unit / tp;
            if (tx < tiles_x) load[((size_t)t * tiles_x + tx) * 3 + p] += n;
          }
        }
      }
    }
    for (size_t k = 0; k < load.size(); ++k)
      if (load[k] > (uint32_t)(k % 3 ? kTileListC : kTileListY)) return;
  }
  plan.tiles_ok = true;
}

}  // namespace

int build_deblock_plan(const h266_picture &pic, const h266_deblock_cu *cus, uint64_t n_cus,
                       const h266_deblock_cu *chroma_cus, uint64_t n_chroma, const h266_deblock_mv_grid *mv,
                       const h266_deblock_params &params, uint32_t cfi, const uint32_t *nf_cols, uint64_t n_cols,
                       const uint32_t *nf_rows, uint64_t n_rows, DeblockPlan &plan, TaskPool *pool) {
  for (int d = 0; d < 2; ++d) {
    plan.segs[d].clear();
    plan.comp[d].assign(1, 0);  // component offsets end with the total count
    plan.max_comp_len[d] = 0;
  }
  if (params.disabled) {
    index_bands(pic, plan);
    index_tiles(pic, cfi, plan);
    return H266_OK;
  }
  for (int d = 0; d < 2; ++d) plan.comp[d].clear();
  if (params.bit_depth < 8 || params.bit_depth > 16)
    return set_error(H266_ERR_INVALID_ARGUMENT, "deblock: bit_depth must be 8..16");
  if (params.ctb_log2_size_y > 16) return set_error(H266_ERR_INVALID_ARGUMENT, "deblock: ctb_log2_size_y too large");
  if (n_cus > (uint64_t)INT32_MAX || n_chroma > (uint64_t)INT32_MAX)
    return set_error(H266_ERR_UNSUPPORTED, "deblock: more than 2^31 - 1 CUs");
  const h266_deblock_cu *lists[2] = {cus, chroma_cus};
  const uint64_t counts[2] = {n_cus, n_chroma};
  for (int l = 0; l < 2; ++l)
    for (uint64_t i = 0; i < counts[l]; ++i) {
      const h266_deblock_cu &c = lists[l][i];
      // Segment bands are 4-line aligned; every VVC CU lies on the 4x4 grid.
      if ((c.x | c.y | c.w | c.h) & 3 || c.w == 0 || c.h == 0)
        return set_error(H266_ERR_UNSUPPORTED, "deblock: CU position/size not on the 4x4 luma grid");
      if ((uint64_t)c.x + c.w > 65535 || (uint64_t)c.y + c.h > 65535)
        return set_error(H266_ERR_UNSUPPORTED, "deblock: CU beyond 65535 samples");
      if (c.has_tb_split && (c.tb_split.n_bounds < 1 || c.tb_split.n_bounds > 3))
        return set_error(H266_ERR_INVALID_ARGUMENT, "deblock: tb_split.n_bounds must be 1..3");
    }
  const int bd = (int)params.bit_depth;
  const uint32_t ctb = 1u << params.ctb_log2_size_y;
  const int pw = (int)pic.luma.width, ph = (int)pic.luma.height;
  MvGrid mvg{mv}, none{nullptr};
  // Six independent lists: (luma, cb, cr) x (vertical, horizontal) pass.  Each
  // is walked and grouped on its own (in parallel with a pool) and the lists
  // are concatenated per pass in plane order.
  const bool sep = chroma_cus != nullptr;
  const int n_lists = cfi != 0 ? 6 : 2;
  thread_local std::vector<int32_t> grid_luma, grid_chroma;
  Walker luma(cus, n_cus, pw, ph, grid_luma);
  std::unique_ptr<Walker> cwalk;
  if (cfi != 0 && sep) cwalk.reset(new Walker(chroma_cus, n_chroma, pw, ph, grid_chroma));
  const Walker &cw = sep && cfi != 0 ? *cwalk : luma;
  const PlaneCfg cfg[3] = {
      {0, 1, 1, params.luma_beta_offset_div2, params.luma_tc_offset_div2, 0, bd, ctb},
      {1, 2, 2, params.cb_beta_offset_div2, params.cb_tc_offset_div2, params.chroma_qp_offset_cb, bd, ctb},
      {2, 2, 2, params.cr_beta_offset_div2, params.cr_tc_offset_div2, params.chroma_qp_offset_cr, bd, ctb}};
  auto one_list = [&](size_t l) {
    thread_local std::vector<Emitted> em;
    thread_local GroupScratch gs;
    const int plane = (int)l / 2, d = (int)l % 2;
    em.clear();
    (plane == 0 ? luma : cw).walk(cfg[plane], d == 0, plane == 0 ? mvg : none, d == 0 ? nf_cols : nf_rows,
                                  d == 0 ? n_cols : n_rows, em);
    DeblockPlan::Part &part = plan.parts[l];
    part.segs.clear();
    part.comp.clear();
    part.max_len = 0;
    group(em, part.segs, part.comp, part.max_len, gs);
  };
  if (pool && pool->size() > 1)
    pool->run((size_t)n_lists, one_list);
  else
    for (int l = 0; l < n_lists; ++l) one_list((size_t)l);
  for (int d = 0; d < 2; ++d) {
    size_t total = 0, total_c = 0;
    for (int l = d; l < n_lists; l += 2) {
      total += plan.parts[l].segs.size();
      total_c += plan.parts[l].comp.size();
    }
    plan.segs[d].reserve(total);
    plan.comp[d].reserve(total_c + 1);
    for (int l = d; l < n_lists; l += 2) {
      const uint32_t base = (uint32_t)plan.segs[d].size();
      const DeblockPlan::Part &part = plan.parts[l];
      plan.segs[d].insert(plan.segs[d].end(), part.segs.begin(), part.segs.end());
      for (uint32_t c : part.comp) plan.comp[d].push_back(base + c);
      plan.max_comp_len[d] = std::max(plan.max_comp_len[d], part.max_len);
    }
    plan.comp[d].push_back((uint32_t)plan.segs[d].size());
  }
  index_bands(pic, plan);
  index_tiles(pic, cfi, plan);
  return H266_OK;
}

// ===================================================================== device
namespace {

// Sample access of the segment filters: reads clamp into the plane (the
// reference's clamped `sample()`), writes outside the plane are dropped and
// written values are Clip1'd.
struct GlobalView {  // a plane in global memory
  DPlane p;
  __host__ __device__ __forceinline__ int rd(int x, int y) const {
    x = min(max(x, 0), p.w - 1);
    y = min(max(y, 0), p.h - 1);
    return p.s[(int64_t)y * p.stride + x];
  }
  __host__ __device__ __forceinline__ void wr(int x, int y, int v, int maxv) const {
    if (x < 0 || y < 0 || x >= p.w || y >= p.h) return;
    p.s[(int64_t)y * p.stride + x] = (uint16_t)min(max(v, 0), maxv);
  }
};

// A window of a plane staged in shared memory: columns [ox, ox + ww) and rows
// [oy, oy + wh) of a w x h plane, `ld` samples per row.  Every clamped
// coordinate a segment of the window's bands touches lies inside the window
// (bands are whole rows / full-height column strips); the window clamp below
// only keeps shared-memory accesses in bounds whatever the input.
struct SharedView {
  uint16_t *s;
  int ld, ox, oy, ww, wh, w, h;
  __host__ __device__ __forceinline__ int rd(int x, int y) const {
    x = min(max(min(max(x, 0), w - 1), ox), ox + ww - 1);
    y = min(max(min(max(y, 0), h - 1), oy), oy + wh - 1);
    return s[(y - oy) * ld + (x - ox)];
  }
  __host__ __device__ __forceinline__ void wr(int x, int y, int v, int maxv) const {
    if (x < 0 || y < 0 || x >= w || y >= h) return;
    if (x < ox || y < oy || x >= ox + ww || y >= oy + wh) return;
    s[(y - oy) * ld + (x - ox)] = (uint16_t)min(max(v, 0), maxv);
  }
};

__host__ __device__ __forceinline__ int clampd(int v, int lo, int hi) { return min(max(v, lo), hi); }

// Long-filter weights of eqs. 1395-1408 as closed forms of the tables
// F7 = {59, 50, 41, 32, 23, 14, 5}, F5 = {58, 45, 32, 19, 6}, F3 = {53, 32, 11}
// and T7 = {6, 5, 4, 3, 2, 1, 1}, T5 = {6, 5, 4, 3, 2}, T3 = {6, 4, 2}, so that
// a fully unrolled filter needs no indexed table.
__host__ __device__ __forceinline__ int long_f(int m, int i) {
  return m == 7 ? 59 - 9 * i : (m == 5 ? 58 - 13 * i : 53 - 21 * i);
}
__host__ __device__ __forceinline__ int long_t(int m, int i) {
  return m == 7 ? (i < 6 ? 6 - i : 1) : (m == 5 ? 6 - i : 6 - 2 * i);
}

// One luma edge segment: §8.8.3.6.2 decision + §8.8.3.6.7 / .8 filters
// (luma_edge_decision / run_luma_filter / short_luma_apply / long_luma_apply,
// src/deblock.rs:1224-1776).  The decision reads lines 0 and 3 before any
// write; every line is then filtered from its own samples and written back
// before the next line is read (lines are disjoint; a line clamped onto
// another one lies outside the plane, so its writes are dropped).  Every
// array index is a compile-time constant after unrolling, so the samples stay
// in registers.
template <class View>
__host__ __device__ void luma_segment(const View &P, const EdgeSeg &e, int maxv) {
  const bool vert = e.flags & 1;
  const int tc = e.tc, beta = e.beta;
  int mp = e.mfl >> 4, mq = e.mfl & 15;
  const int cx = e.x, cy = e.y;
  const bool plt_p = e.flags & 4, plt_q = e.flags & 8;
  // l0[8 + d], l3[8 + d]: lines 0 and 3 at distance d from q0
  int l0[16], l3[16];
#pragma unroll
  for (int d = -8; d < 8; ++d) {
    l0[8 + d] = vert ? P.rd(cx + d, cy) : P.rd(cx, cy + d);
    l3[8 + d] = vert ? P.rd(cx + d, cy + 3) : P.rd(cx + 3, cy + d);
  }
#define P0(i) l0[7 - (i)]
#define Q0(j) l0[8 + (j)]
#define P3(i) l3[7 - (i)]
#define Q3(j) l3[8 + (j)]
  const int dp0 = abs(P0(2) - 2 * P0(1) + P0(0)), dp3 = abs(P3(2) - 2 * P3(1) + P3(0));
  const int dq0 = abs(Q0(2) - 2 * Q0(1) + Q0(0)), dq3 = abs(Q3(2) - 2 * Q3(1) + Q3(0));
  const int sp0 = abs(P0(3) - P0(0)), sq0 = abs(Q0(0) - Q0(3)), spq0 = abs(P0(0) - Q0(0));
  const int sp3 = abs(P3(3) - P3(0)), sq3 = abs(Q3(0) - Q3(3)), spq3 = abs(P3(0) - Q3(0));
  const int tc_gate = (5 * tc + 1) >> 1;
  const bool p_large = mp > 3 && !(e.flags & 2);
  const bool q_large = mq > 3;
  bool long_ok = false;
  if (p_large || q_large) {
    int dp0l = dp0, dp3l = dp3, dq0l = dq0, dq3l = dq3;
    if (p_large) {
      dp0l = (dp0 + abs(P0(5) - 2 * P0(4) + P0(3)) + 1) >> 1;
      dp3l = (dp3 + abs(P3(5) - 2 * P3(4) + P3(3)) + 1) >> 1;
    } else {
      mp = 3;
    }
    if (q_large) {
      dq0l = (dq0 + abs(Q0(5) - 2 * Q0(4) + Q0(3)) + 1) >> 1;
      dq3l = (dq3 + abs(Q3(5) - 2 * Q3(4) + Q3(3)) + 1) >> 1;
    }
    int sp0l = sp0, sp3l = sp3, sq0l = sq0, sq3l = sq3;
    if (mp == 7) {
      sp0l += abs(P0(7) - P0(6) - P0(5) + P0(4));
      sp3l += abs(P3(7) - P3(6) - P3(5) + P3(4));
    }
    if (mq == 7) {
      sq0l += abs(Q0(4) - Q0(5) - Q0(6) + Q0(7));
      sq3l += abs(Q3(4) - Q3(5) - Q3(6) + Q3(7));
    }
    if ((dp0l + dq0l) + (dp3l + dq3l) < beta) {
      const int t1 = (3 * beta) >> 5, t2 = beta >> 4;
      // P(mp) / Q(mq) of lines 0 and 3 (mp, mq in {3, 5, 7})
      const int pm0 = mp == 7 ? P0(7) : (mp == 5 ? P0(5) : P0(3)), pm3 = mp == 7 ? P3(7) : (mp == 5 ? P3(5) : P3(3));
      const int qm0 = mq == 7 ? Q0(7) : (mq == 5 ? Q0(5) : Q0(3)), qm3 = mq == 7 ? Q3(7) : (mq == 5 ? Q3(5) : Q3(3));
      int spl0 = sp0l, sql0 = sq0l, spl3 = sp3l, sql3 = sq3l;
      if (p_large) {
        spl0 = (spl0 + abs(P0(3) - pm0) + 1) >> 1;
        spl3 = (spl3 + abs(P3(3) - pm3) + 1) >> 1;
      }
      if (q_large) {
        sql0 = (sql0 + abs(Q0(3) - qm0) + 1) >> 1;
        sql3 = (sql3 + abs(Q3(3) - qm3) + 1) >> 1;
      }
      long_ok = 2 * (dp0l + dq0l) < t2 && spl0 + sql0 < t1 && spq0 < tc_gate && 2 * (dp3l + dq3l) < t2 &&
                spl3 + sql3 < t1 && spq3 < tc_gate;
    }
  }
#undef P0
#undef Q0
#undef P3
#undef Q3
  if (long_ok) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      // p[i], q[j]: line k; entries beyond mflP / mflQ are zero as in the reference's arrays
      int p[8], q[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int pi = k == 0 ? l0[7 - i] : (k == 3 ? l3[7 - i] : (vert ? P.rd(cx - 1 - i, cy + k) : P.rd(cx + k, cy - 1 - i)));
        const int qi = k == 0 ? l0[8 + i] : (k == 3 ? l3[8 + i] : (vert ? P.rd(cx + i, cy + k) : P.rd(cx + k, cy + i)));
        p[i] = i <= mp ? pi : 0;
        q[i] = i <= mq ? qi : 0;
      }
      int mid;  // refMiddle, eqs. 1389-1394
      if (mp == 5 && mq == 5)
        mid = (p[4] + p[3] + 2 * (p[2] + p[1] + p[0] + q[0] + q[1] + q[2]) + q[3] + q[4] + 8) >> 4;
      else if (mp == mq)
        mid = (p[6] + p[5] + p[4] + p[3] + p[2] + p[1] + 2 * (p[0] + q[0]) + q[1] + q[2] + q[3] + q[4] + q[5] + q[6] +
               8) >> 4;
      else if ((mp == 7 && mq == 5) || (mp == 5 && mq == 7))
        mid = (p[5] + p[4] + p[3] + p[2] + 2 * (p[1] + p[0] + q[0] + q[1]) + q[2] + q[3] + q[4] + q[5] + 8) >> 4;
      else if ((mp == 5 && mq == 3) || (mp == 3 && mq == 5))
        mid = (p[3] + p[2] + p[1] + p[0] + q[0] + q[1] + q[2] + q[3] + 4) >> 3;
      else if (mp == 3 && mq == 7)
        mid = (2 * (p[2] + p[1] + p[0] + q[0]) + p[0] + p[1] + q[1] + q[2] + q[3] + q[4] + q[5] + q[6] + 8) >> 4;
      else
        mid = (p[6] + p[5] + p[4] + p[3] + p[2] + p[1] + 2 * (q[2] + q[1] + q[0] + p[0]) + q[0] + q[1] + 8) >> 4;
      // refP / refQ, eqs. 1395-1396
      const int rp = mp == 7 ? (p[7] + p[6] + 1) >> 1 : (mp == 5 ? (p[5] + p[4] + 1) >> 1 : (p[3] + p[2] + 1) >> 1);
      const int rq = mq == 7 ? (q[7] + q[6] + 1) >> 1 : (mq == 5 ? (q[5] + q[4] + 1) >> 1 : (q[3] + q[2] + 1) >> 1);
#pragma unroll
      for (int i = 0; i < 7; ++i) {
        if (i < mp && !plt_p) {
          const int f = long_f(mp, i), lim = (tc * long_t(mp, i)) >> 1;
          const int v = clampd((mid * f + rp * (64 - f) + 32) >> 6, p[i] - lim, p[i] + lim);
          if (vert) P.wr(cx - i - 1, cy + k, v, maxv);
          else P.wr(cx + k, cy - i - 1, v, maxv);
        }
        if (i < mq && !plt_q) {
          const int f = long_f(mq, i), lim = (tc * long_t(mq, i)) >> 1;
          const int v = clampd((mid * f + rq * (64 - f) + 32) >> 6, q[i] - lim, q[i] + lim);
          if (vert) P.wr(cx + i, cy + k, v, maxv);
          else P.wr(cx + k, cy + i, v, maxv);
        }
      }
    }
    return;
  }
  const int d = dp0 + dq0 + dp3 + dq3;
  if (d >= beta) return;  // dE = 0
  bool strong = false;
  if (mp > 2 && mq > 2) {
    const int t1 = beta >> 3, t2 = beta >> 2;
    strong = 2 * (dp0 + dq0) < t2 && sp0 + sq0 < t1 && spq0 < tc_gate && 2 * (dp3 + dq3) < t2 &&
             sp3 + sq3 < t1 && spq3 < tc_gate;
  }
  if (strong) mp = mq = 3;
  const int side_gate = (beta + (beta >> 1)) >> 3;
  const bool dep = mp > 1 && mq > 1 && dp0 + dp3 < side_gate;
  const bool deq = mp > 1 && mq > 1 && dq0 + dq3 < side_gate;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    int s[8];  // p3 p2 p1 p0 q0 q1 q2 q3 of line k
#pragma unroll
    for (int t = 0; t < 8; ++t)
      s[t] = k == 0 ? l0[4 + t] : (k == 3 ? l3[4 + t] : (vert ? P.rd(cx - 4 + t, cy + k) : P.rd(cx + k, cy - 4 + t)));
    const int p3 = s[0], p2 = s[1], p1 = s[2], p0 = s[3], q0 = s[4], q1 = s[5], q2 = s[6], q3 = s[7];
    int np = 0, nq = 0;  // samples written this line, from p0 / q0 outwards
    int op0 = 0, op1 = 0, op2 = 0, oq0 = 0, oq1 = 0, oq2 = 0;
    if (strong) {
      op0 = clampd((p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3, p0 - 3 * tc, p0 + 3 * tc);
      op1 = clampd((p2 + p1 + p0 + q0 + 2) >> 2, p1 - 2 * tc, p1 + 2 * tc);
      op2 = clampd((2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3, p2 - tc, p2 + tc);
      oq0 = clampd((p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3, q0 - 3 * tc, q0 + 3 * tc);
      oq1 = clampd((p0 + q0 + q1 + q2 + 2) >> 2, q1 - 2 * tc, q1 + 2 * tc);
      oq2 = clampd((p0 + q0 + q1 + 3 * q2 + 2 * q3 + 4) >> 3, q2 - tc, q2 + tc);
      np = nq = 3;
    } else {
      const int raw = (9 * (q0 - p0) - 3 * (q1 - p1) + 8) >> 4;
      if (abs(raw) < tc * 10) {
        const int delta = clampd(raw, -tc, tc);
        op0 = p0 + delta;
        oq0 = q0 - delta;
        np = nq = 1;
        if (dep) {
          op1 = p1 + clampd((((p2 + p0 + 1) >> 1) - p1 + delta) >> 1, -(tc >> 1), tc >> 1);
          np = 2;
        }
        if (deq) {
          oq1 = q1 + clampd((((q2 + q0 + 1) >> 1) - q1 - delta) >> 1, -(tc >> 1), tc >> 1);
          nq = 2;
        }
      }
    }
    if (plt_p) np = 0;
    if (plt_q) nq = 0;
    const int op[3] = {op0, op1, op2}, oq[3] = {oq0, oq1, oq2};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (i < np) {
        if (vert) P.wr(cx - i - 1, cy + k, op[i], maxv);
        else P.wr(cx + k, cy - i - 1, op[i], maxv);
      }
      if (i < nq) {
        if (vert) P.wr(cx + i, cy + k, oq[i], maxv);
        else P.wr(cx + k, cy + i, oq[i], maxv);
      }
    }
  }
}

// One chroma edge segment (2 lines): run_chroma_filter_v / _h with the strong
// decision and filters of src/deblock.rs:1803-2075.  Constant indices only.
template <class View>
__host__ __device__ void chroma_segment(const View &P, const EdgeSeg &e, int maxv) {
  const bool vert = e.flags & 1;
  const int tc = e.tc, beta = e.beta, mp = e.mfl >> 4, mq = e.mfl & 15;
  const int cx = e.x, cy = e.y;
  const bool plt_p = e.flags & 4, plt_q = e.flags & 8;
  int v[2][8];  // v[k][4 + d], d in [-4, 3]
#pragma unroll
  for (int k = 0; k < 2; ++k)
#pragma unroll
    for (int d = -4; d < 4; ++d) v[k][4 + d] = vert ? P.rd(cx + d, cy + k) : P.rd(cx + k, cy + d);
  const bool eligible = vert ? (mp == 3 && mq == 3) : (mq == 3 && (mp == 3 || mp == 1));
  const bool short_p = !vert && mp == 1;
  if (eligible) {
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int p1 = v[k][2], p0 = v[k][3], q0 = v[k][4], q1 = v[k][5], q2 = v[k][6], q3 = v[k][7];
      const int p3 = short_p ? p1 : v[k][0], p2 = short_p ? p1 : v[k][1];
      const int dpq = 2 * (abs(p2 - 2 * p1 + p0) + abs(q2 - 2 * q1 + q0));
      ok = ok && dpq < (beta >> 2) && abs(p3 - p0) + abs(q0 - q3) < (beta >> 3) && abs(p0 - q0) < ((5 * tc + 1) >> 1);
    }
    if (ok) {
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int p3 = v[k][0], p2 = v[k][1], p1 = v[k][2], p0 = v[k][3];
        const int q0 = v[k][4], q1 = v[k][5], q2 = v[k][6], q3 = v[k][7];
        int op[3] = {0, 0, 0}, oq[3];
        int np;
        if (short_p) {
          op[0] = clampd((3 * p1 + 2 * p0 + q0 + q1 + q2 + 4) >> 3, p0 - tc, p0 + tc);
          oq[0] = clampd((2 * p1 + p0 + 2 * q0 + q1 + q2 + q3 + 4) >> 3, q0 - tc, q0 + tc);
          np = 1;
        } else {
          op[0] = clampd((p3 + p2 + p1 + 2 * p0 + q0 + q1 + q2 + 4) >> 3, p0 - tc, p0 + tc);
          op[1] = clampd((2 * p3 + p2 + 2 * p1 + p0 + q0 + q1 + 4) >> 3, p1 - tc, p1 + tc);
          op[2] = clampd((3 * p3 + 2 * p2 + p1 + p0 + q0 + 4) >> 3, p2 - tc, p2 + tc);
          oq[0] = clampd((p2 + p1 + p0 + 2 * q0 + q1 + q2 + q3 + 4) >> 3, q0 - tc, q0 + tc);
          np = 3;
        }
        oq[1] = clampd((p1 + p0 + q0 + 2 * q1 + q2 + 2 * q3 + 4) >> 3, q1 - tc, q1 + tc);
        oq[2] = clampd((p0 + q0 + q1 + 2 * q2 + 3 * q3 + 4) >> 3, q2 - tc, q2 + tc);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          if (!plt_p && i < np) {
            if (vert) P.wr(cx - i - 1, cy + k, op[i], maxv);
            else P.wr(cx + k, cy - i - 1, op[i], maxv);
          }
          if (!plt_q) {
            if (vert) P.wr(cx + i, cy + k, oq[i], maxv);
            else P.wr(cx + k, cy + i, oq[i], maxv);
          }
        }
      }
      return;
    }
  }
#pragma unroll
  for (int k = 0; k < 2; ++k) {  // weak filter, eqs. 1421-1423
    const int p1 = v[k][2], p0 = v[k][3], q0 = v[k][4], q1 = v[k][5];
    const int delta = clampd(((q0 - p0) * 4 + p1 - q1 + 4) >> 3, -tc, tc);
    if (!plt_p) {
      if (vert) P.wr(cx - 1, cy + k, p0 + delta, maxv);
      else P.wr(cx + k, cy - 1, p0 + delta, maxv);
    }
    if (!plt_q) {
      if (vert) P.wr(cx, cy + k, q0 - delta, maxv);
      else P.wr(cx + k, cy, q0 - delta, maxv);
    }
  }
}

// ------------------------------------------------------------ line-parallel segments
// The strip kernels filter a segment with one lane per line (4 luma, 2 chroma
// lines): each lane loads its line, the decision terms of lines 0 and 3 (luma)
// or of both lines (chroma) are exchanged between the lanes of the group, and
// each lane filters and writes its own line.  The arithmetic is that of
// luma_segment / chroma_segment above, split into per-line pieces; every line
// is loaded before any line is written, as there.

// Access to one line of a segment by distance d from its q0 sample (negative
// on the P side): through a clamping view, or -- when the segment's samples
// lie inside the staged window -- straight in shared memory with the step SN
// between samples along the edge normal.
template <class View>
struct ClampLine {
  const View &P;
  int qx, qy;  // q0 of the line
  bool vert;
  __host__ __device__ __forceinline__ int rd(int d) const { return vert ? P.rd(qx + d, qy) : P.rd(qx, qy + d); }
  __host__ __device__ __forceinline__ void wr(int d, int v, int maxv) const {
    if (vert) P.wr(qx + d, qy, v, maxv);
    else P.wr(qx, qy + d, v, maxv);
  }
};
template <int SN>
struct RawLine {
  uint16_t *q;  // q0 of the line
  __host__ __device__ __forceinline__ int rd(int d) const { return q[d * SN]; }
  __host__ __device__ __forceinline__ void wr(int d, int v, int maxv) const { q[d * SN] = (uint16_t)min(max(v, 0), maxv); }
};
struct RawLineDyn {
  uint16_t *q;
  int sn;
  __host__ __device__ __forceinline__ int rd(int d) const { return q[d * sn]; }
  __host__ __device__ __forceinline__ void wr(int d, int v, int maxv) const { q[d * sn] = (uint16_t)min(max(v, 0), maxv); }
};

// Samples of a luma line: s[8 + d] at distance d from q0, d in [-8, 7].
template <class Line>
__host__ __device__ __forceinline__ void load_luma_line(const Line &L, int s[16]) {
#pragma unroll
  for (int d = -8; d < 8; ++d) s[8 + d] = L.rd(d);
}

// The decision terms of one luma line (§8.8.3.6.2, src/deblock.rs:1224-1410).
struct LumaStats {
  int dp, dq, sp, sq, spq;  // |p2-2p1+p0|, |q2-2q1+q0|, |p3-p0|, |q0-q3|, |p0-q0|
  int dpx, dqx;             // |p5-2p4+p3|, |q5-2q4+q3|
  int sp7, sq7;             // |p7-p6-p5+p4|, |q4-q5-q6+q7|
  int pmd, qmd;             // |p3-p(mflP)|, |q3-q(mflQ)| for mfl 5 / 7
};

__host__ __device__ __forceinline__ LumaStats luma_stats(const EdgeSeg &e, const int s[16]) {
#define PL(i) s[7 - (i)]
#define QL(j) s[8 + (j)]
  const int mp = e.mfl >> 4, mq = e.mfl & 15;
  LumaStats t;
  t.dp = abs(PL(2) - 2 * PL(1) + PL(0));
  t.dq = abs(QL(2) - 2 * QL(1) + QL(0));
  t.sp = abs(PL(3) - PL(0));
  t.sq = abs(QL(0) - QL(3));
  t.spq = abs(PL(0) - QL(0));
  t.dpx = abs(PL(5) - 2 * PL(4) + PL(3));
  t.dqx = abs(QL(5) - 2 * QL(4) + QL(3));
  t.sp7 = abs(PL(7) - PL(6) - PL(5) + PL(4));
  t.sq7 = abs(QL(4) - QL(5) - QL(6) + QL(7));
  t.pmd = abs(PL(3) - (mp == 7 ? PL(7) : (mp == 5 ? PL(5) : PL(3))));
  t.qmd = abs(QL(3) - (mq == 7 ? QL(7) : (mq == 5 ? QL(5) : QL(3))));
#undef PL
#undef QL
  return t;
}

struct LumaDecision {
  int mode;  // 0: no filtering (dE = 0), 1: long filter, 2: short filter
  int mp, mq;
  bool strong, dep, deq;
};

// The segment's decision from the terms of lines 0 (a) and 3 (b).
__host__ __device__ __forceinline__ LumaDecision luma_decide(const EdgeSeg &e, const LumaStats &a,
                                                             const LumaStats &b) {
  const int tc = e.tc, beta = e.beta;
  LumaDecision dc;
  dc.mp = e.mfl >> 4;
  dc.mq = e.mfl & 15;
  dc.strong = dc.dep = dc.deq = false;
  const int tc_gate = (5 * tc + 1) >> 1;
  const bool p_large = dc.mp > 3 && !(e.flags & 2);
  const bool q_large = dc.mq > 3;
  if (p_large || q_large) {
    int dp0l = a.dp, dp3l = b.dp, dq0l = a.dq, dq3l = b.dq;
    if (p_large) {
      dp0l = (a.dp + a.dpx + 1) >> 1;
      dp3l = (b.dp + b.dpx + 1) >> 1;
    } else {
      dc.mp = 3;
    }
    if (q_large) {
      dq0l = (a.dq + a.dqx + 1) >> 1;
      dq3l = (b.dq + b.dqx + 1) >> 1;
    }
    int sp0l = a.sp, sp3l = b.sp, sq0l = a.sq, sq3l = b.sq;
    if (dc.mp == 7) {
      sp0l += a.sp7;
      sp3l += b.sp7;
    }
    if (dc.mq == 7) {
      sq0l += a.sq7;
      sq3l += b.sq7;
    }
    if ((dp0l + dq0l) + (dp3l + dq3l) < beta) {
      const int t1 = (3 * beta) >> 5, t2 = beta >> 4;
      int spl0 = sp0l, sql0 = sq0l, spl3 = sp3l, sql3 = sq3l;
      if (p_large) {
        spl0 = (spl0 + a.pmd + 1) >> 1;
        spl3 = (spl3 + b.pmd + 1) >> 1;
      }
      if (q_large) {
        sql0 = (sql0 + a.qmd + 1) >> 1;
        sql3 = (sql3 + b.qmd + 1) >> 1;
      }
      if (2 * (dp0l + dq0l) < t2 && spl0 + sql0 < t1 && a.spq < tc_gate && 2 * (dp3l + dq3l) < t2 &&
          spl3 + sql3 < t1 && b.spq < tc_gate) {
        dc.mode = 1;
        return dc;
      }
    }
  }
  if (a.dp + a.dq + b.dp + b.dq >= beta) {
    dc.mode = 0;  // dE = 0
    return dc;
  }
  dc.mode = 2;
  if (dc.mp > 2 && dc.mq > 2) {
    const int t1 = beta >> 3, t2 = beta >> 2;
    dc.strong = 2 * (a.dp + a.dq) < t2 && a.sp + a.sq < t1 && a.spq < tc_gate && 2 * (b.dp + b.dq) < t2 &&
                b.sp + b.sq < t1 && b.spq < tc_gate;
  }
  if (dc.strong) dc.mp = dc.mq = 3;
  const int side_gate = (beta + (beta >> 1)) >> 3;
  dc.dep = dc.mp > 1 && dc.mq > 1 && a.dp + b.dp < side_gate;
  dc.deq = dc.mp > 1 && dc.mq > 1 && a.dq + b.dq < side_gate;
  return dc;
}

// Filters one luma line (samples s) of a segment after its decision.
template <class Line>
__host__ __device__ __forceinline__ void luma_filter_line(const Line &L, const EdgeSeg &e, const LumaDecision &dc,
                                                          const int s[16], int maxv) {
  const int tc = e.tc, mp = dc.mp, mq = dc.mq;
  const bool plt_p = e.flags & 4, plt_q = e.flags & 8;
  if (dc.mode == 1) {
    int p[8], q[8];  // entries beyond mflP / mflQ are zero as in the reference's arrays
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      p[i] = i <= mp ? s[7 - i] : 0;
      q[i] = i <= mq ? s[8 + i] : 0;
    }
    int mid;  // refMiddle, eqs. 1389-1394
    if (mp == 5 && mq == 5)
      mid = (p[4] + p[3] + 2 * (p[2] + p[1] + p[0] + q[0] + q[1] + q[2]) + q[3] + q[4] + 8) >> 4;
    else if (mp == mq)
      mid = (p[6] + p[5] + p[4] + p[3] + p[2] + p[1] + 2 * (p[0] + q[0]) + q[1] + q[2] + q[3] + q[4] + q[5] + q[6] +
             8) >> 4;
    else if ((mp == 7 && mq == 5) || (mp == 5 && mq == 7))
      mid = (p[5] + p[4] + p[3] + p[2] + 2 * (p[1] + p[0] + q[0] + q[1]) + q[2] + q[3] + q[4] + q[5] + 8) >> 4;
    else if ((mp == 5 && mq == 3) || (mp == 3 && mq == 5))
      mid = (p[3] + p[2] + p[1] + p[0] + q[0] + q[1] + q[2] + q[3] + 4) >> 3;
    else if (mp == 3 && mq == 7)
      mid = (2 * (p[2] + p[1] + p[0] + q[0]) + p[0] + p[1] + q[1] + q[2] + q[3] + q[4] + q[5] + q[6] + 8) >> 4;
    else
      mid = (p[6] + p[5] + p[4] + p[3] + p[2] + p[1] + 2 * (q[2] + q[1] + q[0] + p[0]) + q[0] + q[1] + 8) >> 4;
    const int rp = mp == 7 ? (p[7] + p[6] + 1) >> 1 : (mp == 5 ? (p[5] + p[4] + 1) >> 1 : (p[3] + p[2] + 1) >> 1);
    const int rq = mq == 7 ? (q[7] + q[6] + 1) >> 1 : (mq == 5 ? (q[5] + q[4] + 1) >> 1 : (q[3] + q[2] + 1) >> 1);
#pragma unroll
    for (int i = 0; i < 7; ++i) {
      if (i < mp && !plt_p) {
        const int f = long_f(mp, i), lim = (tc * long_t(mp, i)) >> 1;
        L.wr(-i - 1, clampd((mid * f + rp * (64 - f) + 32) >> 6, p[i] - lim, p[i] + lim), maxv);
      }
      if (i < mq && !plt_q) {
        const int f = long_f(mq, i), lim = (tc * long_t(mq, i)) >> 1;
        L.wr(i, clampd((mid * f + rq * (64 - f) + 32) >> 6, q[i] - lim, q[i] + lim), maxv);
      }
    }
    return;
  }
  if (dc.mode == 0) return;
  const int p3 = s[4], p2 = s[5], p1 = s[6], p0 = s[7], q0 = s[8], q1 = s[9], q2 = s[10], q3 = s[11];
  int np = 0, nq = 0;
  int op0 = 0, op1 = 0, op2 = 0, oq0 = 0, oq1 = 0, oq2 = 0;
  if (dc.strong) {
    op0 = clampd((p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3, p0 - 3 * tc, p0 + 3 * tc);
    op1 = clampd((p2 + p1 + p0 + q0 + 2) >> 2, p1 - 2 * tc, p1 + 2 * tc);
    op2 = clampd((2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3, p2 - tc, p2 + tc);
    oq0 = clampd((p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3, q0 - 3 * tc, q0 + 3 * tc);
    oq1 = clampd((p0 + q0 + q1 + q2 + 2) >> 2, q1 - 2 * tc, q1 + 2 * tc);
    oq2 = clampd((p0 + q0 + q1 + 3 * q2 + 2 * q3 + 4) >> 3, q2 - tc, q2 + tc);
    np = nq = 3;
  } else {
    const int raw = (9 * (q0 - p0) - 3 * (q1 - p1) + 8) >> 4;
    if (abs(raw) < tc * 10) {
      const int delta = clampd(raw, -tc, tc);
      op0 = p0 + delta;
      oq0 = q0 - delta;
      np = nq = 1;
      if (dc.dep) {
        op1 = p1 + clampd((((p2 + p0 + 1) >> 1) - p1 + delta) >> 1, -(tc >> 1), tc >> 1);
        np = 2;
      }
      if (dc.deq) {
        oq1 = q1 + clampd((((q2 + q0 + 1) >> 1) - q1 - delta) >> 1, -(tc >> 1), tc >> 1);
        nq = 2;
      }
    }
  }
  if (plt_p) np = 0;
  if (plt_q) nq = 0;
  const int op[3] = {op0, op1, op2}, oq[3] = {oq0, oq1, oq2};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (i < np) L.wr(-i - 1, op[i], maxv);
    if (i < nq) L.wr(i, oq[i], maxv);
  }
}

// Samples of a chroma line: s[4 + d], d in [-4, 3].
template <class Line>
__host__ __device__ __forceinline__ void load_chroma_line(const Line &L, int s[8]) {
#pragma unroll
  for (int d = -4; d < 4; ++d) s[4 + d] = L.rd(d);
}

// Whether the segment may take the strong chroma filter (src/deblock.rs:1803-1890).
__host__ __device__ __forceinline__ bool chroma_eligible(const EdgeSeg &e) {
  const int mp = e.mfl >> 4, mq = e.mfl & 15;
  return (e.flags & 1) ? (mp == 3 && mq == 3) : (mq == 3 && (mp == 3 || mp == 1));
}

// The strong-filter condition of one chroma line.
__host__ __device__ __forceinline__ bool chroma_line_ok(const EdgeSeg &e, const int s[8]) {
  const bool short_p = !(e.flags & 1) && (e.mfl >> 4) == 1;
  const int tc = e.tc, beta = e.beta;
  const int p1 = s[2], p0 = s[3], q0 = s[4], q1 = s[5], q2 = s[6], q3 = s[7];
  const int p3 = short_p ? p1 : s[0], p2 = short_p ? p1 : s[1];
  const int dpq = 2 * (abs(p2 - 2 * p1 + p0) + abs(q2 - 2 * q1 + q0));
  return dpq < (beta >> 2) && abs(p3 - p0) + abs(q0 - q3) < (beta >> 3) && abs(p0 - q0) < ((5 * tc + 1) >> 1);
}

// Filters one chroma line: strong when `strong` (eligible and both lines ok), else weak.
template <class Line>
__host__ __device__ __forceinline__ void chroma_filter_line(const Line &L, const EdgeSeg &e, bool strong,
                                                            const int s[8], int maxv) {
  const bool vert = e.flags & 1;
  const int tc = e.tc;
  const bool plt_p = e.flags & 4, plt_q = e.flags & 8;
  const int p3 = s[0], p2 = s[1], p1 = s[2], p0 = s[3], q0 = s[4], q1 = s[5], q2 = s[6], q3 = s[7];
  if (strong) {
    const bool short_p = !vert && (e.mfl >> 4) == 1;
    int op[3] = {0, 0, 0}, oq[3];
    int np;
    if (short_p) {
      op[0] = clampd((3 * p1 + 2 * p0 + q0 + q1 + q2 + 4) >> 3, p0 - tc, p0 + tc);
      oq[0] = clampd((2 * p1 + p0 + 2 * q0 + q1 + q2 + q3 + 4) >> 3, q0 - tc, q0 + tc);
      np = 1;
    } else {
      op[0] = clampd((p3 + p2 + p1 + 2 * p0 + q0 + q1 + q2 + 4) >> 3, p0 - tc, p0 + tc);
      op[1] = clampd((2 * p3 + p2 + 2 * p1 + p0 + q0 + q1 + 4) >> 3, p1 - tc, p1 + tc);
      op[2] = clampd((3 * p3 + 2 * p2 + p1 + p0 + q0 + 4) >> 3, p2 - tc, p2 + tc);
      oq[0] = clampd((p2 + p1 + p0 + 2 * q0 + q1 + q2 + q3 + 4) >> 3, q0 - tc, q0 + tc);
      np = 3;
    }
    oq[1] = clampd((p1 + p0 + q0 + 2 * q1 + q2 + 2 * q3 + 4) >> 3, q1 - tc, q1 + tc);
    oq[2] = clampd((p0 + q0 + q1 + 2 * q2 + 3 * q3 + 4) >> 3, q2 - tc, q2 + tc);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (!plt_p && i < np) L.wr(-i - 1, op[i], maxv);
      if (!plt_q) L.wr(i, oq[i], maxv);
    }
    return;
  }
  const int delta = clampd(((q0 - p0) * 4 + p1 - q1 + 4) >> 3, -tc, tc);  // weak filter, eqs. 1421-1423
  if (!plt_p) L.wr(-1, p0 + delta, maxv);
  if (!plt_q) L.wr(0, q0 - delta, maxv);
}

struct Planes3 {
  DPlane p[3];
};

// Global-memory deblocking: one thread per component.
__global__ void __launch_bounds__(128) k_deblock_components(Planes3 planes, const EdgeSeg *__restrict__ segs,
                                                            const uint32_t *__restrict__ comp, uint32_t n_comp,
                                                            int maxv) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_comp) return;
  const uint32_t b = comp[c], e = comp[c + 1];
  for (uint32_t i = b; i < e; ++i) {
    const EdgeSeg s = segs[i];
    if (s.plane == 0) luma_segment(GlobalView{planes.p[0]}, s, maxv);
    else chroma_segment(GlobalView{planes.p[s.plane]}, s, maxv);
  }
}

// ------------------------------------------------------------ strip kernels
// Every vertical-pass component lies in one band of 4 luma / 2 chroma rows
// (its segments share the band) and every horizontal-pass component in one
// band of 4 / 2 columns, so a CTA that holds whole rows (vertical pass) or a
// full-height column strip (horizontal pass) in shared memory runs its
// components without touching samples of other CTAs.  All clamped reads of a
// segment stay inside the staged window: rows clamp into the plane, whose
// whole width (rows kernel) or height (columns kernel) is staged.
constexpr int kStripCols = 8;              // columns per horizontal-pass CTA (two luma bands)
constexpr int kStripVec = kStripCols / 8;  // 16-byte vectors per strip row
constexpr int kMaxStripSmem = 200 * 1024;  // dynamic shared memory per CTA

struct StripParams {
  DPlane src[3], dst[3];
  EdgeSeg const *segs;
  uint32_t const *comp;
  uint32_t const *band_first;
  uint32_t band_off[3];
  uint32_t n_bands[3];
  uint32_t ctas[3];  // CTAs per plane
  const uint16_t *lut;
  int maxv;
  // Grid mode (side information built on the device): the pass's segments in
  // per-band cell grids, grid[p][band * grid_slots[p] + pos / unit] (bs 0:
  // none), unit 4 luma / 8 chroma samples along the edge normal.
  int grid_mode;
  const EdgeSeg *grid[3];
  uint32_t grid_slots[3], grid_bands[3];
};

// Shared-memory row pitch of the rows kernel: whole 16-byte vectors plus one
// more, so that the four rows of a band start in different banks.
__host__ __device__ __forceinline__ int row_pitch(int w) { return ((w + 7) & ~7) + 8; }

__device__ __forceinline__ bool vec_ok(const DPlane &p) { return ((uintptr_t)p.s & 15) == 0 && (p.stride & 7) == 0; }

__device__ __forceinline__ int plane_of(const StripParams &a, int &bid) {
  int plane = 0;
  while (plane < 2 && bid >= (int)a.ctas[plane]) {
    bid -= (int)a.ctas[plane];
    ++plane;
  }
  return plane;
}

// One segment by a group of G lanes (G = 4 luma lines, 2 chroma lines); lane
// k of the group owns line k.  `base` is the group's first lane in the warp.
// PITCH is the window's row pitch when it is a compile-time constant (0:
// v.ld), used for direct access along columns.
template <int G, class Line>
__device__ __forceinline__ void segment_lines(const Line &L, const EdgeSeg &e, int maxv, int base, unsigned mask) {
  if (G == 4) {
    int s[16];
    load_luma_line(L, s);
    const LumaStats t = luma_stats(e, s);
    LumaStats a, b;  // lines 0 and 3
#define XCHG(f)                       \
  a.f = __shfl_sync(mask, t.f, base); \
  b.f = __shfl_sync(mask, t.f, base + 3);
    XCHG(dp) XCHG(dq) XCHG(sp) XCHG(sq) XCHG(spq) XCHG(dpx) XCHG(dqx) XCHG(sp7) XCHG(sq7) XCHG(pmd) XCHG(qmd)
#undef XCHG
    luma_filter_line(L, e, luma_decide(e, a, b), s, maxv);
  } else {
    int s[8];
    load_chroma_line(L, s);
    const bool ok = chroma_line_ok(e, s);
    const bool both = __shfl_sync(mask, ok, base) && __shfl_sync(mask, ok, base + 1);
    chroma_filter_line(L, e, chroma_eligible(e) && both, s, maxv);
  }
}

template <int G, int PITCH>
__device__ __forceinline__ void segment_group(const SharedView &v, const EdgeSeg &e, int maxv, int k, int base,
                                              unsigned mask) {
  const bool vert = e.flags & 1;
  constexpr int R = G == 4 ? 8 : 4;  // samples read on each side of the edge
  const int qx = vert ? e.x : e.x + k, qy = vert ? e.y + k : e.y;
  // the segment's samples: R on each side across G lines
  const int x0 = vert ? e.x - R : e.x, x1 = vert ? e.x + R : e.x + G;
  const int y0 = vert ? e.y : e.y - R, y1 = vert ? e.y + G : e.y + R;
  const bool inside = x0 >= v.ox && y0 >= v.oy && x1 <= v.ox + v.ww && y1 <= v.oy + v.wh;
  if (inside) {  // uniform over the group: the window lies inside the plane, no clamping
    uint16_t *q = v.s + (qy - v.oy) * v.ld + (qx - v.ox);
    if (vert) segment_lines<G>(RawLine<1>{q}, e, maxv, base, mask);
    else if (PITCH > 0) segment_lines<G>(RawLine<(PITCH > 0 ? PITCH : 1)>{q}, e, maxv, base, mask);
    else segment_lines<G>(RawLineDyn{q, v.ld}, e, maxv, base, mask);
  } else {
    segment_lines<G>(ClampLine<SharedView>{v, qx, qy, vert}, e, maxv, base, mask);
  }
}

// Components [c0, c1) of the window, one lane group per component.  All lanes
// of a group walk the same segments; after each segment the group
// synchronises, as the next segment may read samples another lane wrote
// (a line clamped onto another at the plane edge).
template <int G, int PITCH>
__device__ __forceinline__ void run_components(const StripParams &a, const SharedView &v, uint32_t c0, uint32_t c1) {
  const int lane = threadIdx.x & 31, k = lane % G, base = lane - k;
  const unsigned mask = ((1u << G) - 1) << base;
  const uint32_t groups = blockDim.x / G;
  for (uint32_t c = c0 + threadIdx.x / G; c < c1; c += groups) {
    const uint32_t e = a.comp[c + 1];
    for (uint32_t i = a.comp[c]; i < e; ++i) {
      segment_group<G, PITCH>(v, a.segs[i], a.maxv, k, base, mask);
      __syncwarp(mask);
    }
  }
}

// Grid mode: does the cell at slot s, whose footprint starts at `start`,
// continue a run -- does an earlier footprint of the band end past `start`?
// Footprints [pos - R(mflP), pos + R(mflQ)) reach at most 8 samples and
// cells are 4 (luma) or 8 (chroma) samples apart, so only the 3 cells before
// s can reach it.
__device__ __forceinline__ bool continues_run(const EdgeSeg *cells, uint32_t s, int start) {
  for (uint32_t t = s > 3 ? s - 3 : 0; t < s; ++t) {
    const EdgeSeg f = cells[t];
    if (f.bs && ((f.flags & 1) ? f.x : f.y) + reach_d(f.mfl & 15) > start) return true;
  }
  return false;
}

// Grid mode: the runs of bands [0, nb) of cell grid g (ns cells per band), one
// lane group per run.  A run is a maximal sequence of occupied cells, in
// position order, each starting before the furthest footprint end of the
// cells before it: the host grouping's components, whose members come in
// position order when every row and column of the CU map is in decode order
// (checked on the host before the walk runs on the device).  Footprint starts
// never decrease along a band (spacing 4, reach 4..8), so a run ends at the
// first occupied cell that does not start inside it, and that cell lies
// within 3 cells of the run's last member or not at all.
template <int G, int PITCH>
__device__ __forceinline__ void run_cell_runs(const StripParams &a, const SharedView &v, const EdgeSeg *g, uint32_t ns,
                                              uint32_t nb) {
  const int lane = threadIdx.x & 31, k = lane % G, base = lane - k;
  const unsigned mask = ((1u << G) - 1) << base;
  const uint32_t groups = blockDim.x / G, total = ns * nb;
  for (uint32_t i = threadIdx.x / G; i < total; i += groups) {
    const uint32_t b = i / ns, s = i - b * ns;
    const EdgeSeg *cells = g + (size_t)b * ns;
    EdgeSeg e = cells[s];
    if (!e.bs) continue;
    const bool vert = e.flags & 1;
    int pos = vert ? e.x : e.y;
    if (continues_run(cells, s, pos - reach_d(e.mfl >> 4))) continue;  // not the first of its run
    int end = pos + reach_d(e.mfl & 15);
    uint32_t cur = s;
    for (;;) {
      segment_group<G, PITCH>(v, e, a.maxv, k, base, mask);
      __syncwarp(mask);
      uint32_t nx = cur + 1;
      bool found = false;
      for (; nx < ns && nx <= cur + 3; ++nx) {
        e = cells[nx];
        if (e.bs) {
          found = true;
          break;
        }
      }
      if (!found) break;
      pos = vert ? e.x : e.y;
      if (pos - reach_d(e.mfl >> 4) >= end) break;
      end = max(end, pos + reach_d(e.mfl & 15));
      cur = nx;
    }
  }
}

// Vertical pass: one CTA per band of rows, all planes in one grid.  Loads the
// rows from src (luma through the LMCS LUT), filters, stores them to dst.
__global__ void __launch_bounds__(128) k_deblock_rows(StripParams a) {
  extern __shared__ __align__(16) uint16_t sm[];
  int band = blockIdx.x;
  const int plane = plane_of(a, band);
  const DPlane src = a.src[plane], dst = a.dst[plane];
  const int unit = plane ? 2 : 4;
  const int y0 = band * unit, rows = min(unit, src.h - y0), w = src.w;
  const int ld = row_pitch(w);
  const uint16_t *lut = plane == 0 ? a.lut : nullptr;
  const int nvec = vec_ok(src) ? w / 8 : 0;
  for (int i = threadIdx.x; i < rows * nvec; i += blockDim.x) {
    const int r = i / nvec, c = (i - r * nvec) * 8;
    uint4 q = *reinterpret_cast<const uint4 *>(src.s + (int64_t)(y0 + r) * src.stride + c);
    if (lut) {
      uint32_t *u = reinterpret_cast<uint32_t *>(&q);
#pragma unroll
      for (int k = 0; k < 4; ++k) u[k] = (uint32_t)lut[u[k] & 0xFFFF] | (uint32_t)lut[u[k] >> 16] << 16;
    }
    *reinterpret_cast<uint4 *>(sm + r * ld + c) = q;
  }
  const int tail = w - nvec * 8;
  for (int i = threadIdx.x; i < rows * tail; i += blockDim.x) {
    const int r = i / tail, c = nvec * 8 + (i - r * tail);
    const uint16_t x = src.s[(int64_t)(y0 + r) * src.stride + c];
    sm[r * ld + c] = lut ? lut[x] : x;
  }
  __syncthreads();
  const SharedView view{sm, ld, 0, y0, w, rows, w, src.h};
  if (a.grid_mode) {
    if ((uint32_t)band < a.grid_bands[plane]) {
      const EdgeSeg *g = a.grid[plane] + (size_t)band * a.grid_slots[plane];
      if (plane == 0) run_cell_runs<4, 0>(a, view, g, a.grid_slots[plane], 1);
      else run_cell_runs<2, 0>(a, view, g, a.grid_slots[plane], 1);
    }
  } else {
    const uint32_t *bf = a.band_first + a.band_off[plane];
    if (plane == 0) run_components<4, 0>(a, view, bf[band], bf[band + 1]);
    else run_components<2, 0>(a, view, bf[band], bf[band + 1]);
  }
  __syncthreads();
  const int nvo = vec_ok(dst) ? w / 8 : 0;
  for (int i = threadIdx.x; i < rows * nvo; i += blockDim.x) {
    const int r = i / nvo, c = (i - r * nvo) * 8;
    *reinterpret_cast<uint4 *>(dst.s + (int64_t)(y0 + r) * dst.stride + c) =
        *reinterpret_cast<const uint4 *>(sm + r * ld + c);
  }
  const int tail_o = w - nvo * 8;
  for (int i = threadIdx.x; i < rows * tail_o; i += blockDim.x) {
    const int r = i / tail_o, c = nvo * 8 + (i - r * tail_o);
    dst.s[(int64_t)(y0 + r) * dst.stride + c] = sm[r * ld + c];
  }
}

// Horizontal pass: one CTA per 8-column strip (full plane height), in place.
__global__ void __launch_bounds__(128, 8) k_deblock_cols(StripParams a) {
  extern __shared__ __align__(16) uint16_t sm[];
  int strip = blockIdx.x;
  const int plane = plane_of(a, strip);
  const DPlane p = a.dst[plane];
  const int unit = plane ? 2 : 4;
  const int x0 = strip * kStripCols, cols = min(kStripCols, p.w - x0), h = p.h;
  const bool vec = cols == kStripCols && vec_ok(p);
  if (vec) {
    for (int i = threadIdx.x; i < h * kStripVec; i += blockDim.x) {
      const int r = i / kStripVec, c = (i % kStripVec) * 8;
      *reinterpret_cast<uint4 *>(sm + r * kStripCols + c) =
          *reinterpret_cast<const uint4 *>(p.s + (int64_t)r * p.stride + x0 + c);
    }
  } else {
    for (int i = threadIdx.x; i < h * cols; i += blockDim.x) {
      const int r = i / cols, c = i - r * cols;
      sm[r * kStripCols + c] = p.s[(int64_t)r * p.stride + x0 + c];
    }
  }
  __syncthreads();
  const SharedView view{sm, kStripCols, x0, 0, cols, h, p.w, h};
  if (a.grid_mode) {
    const uint32_t nb = a.grid_bands[plane];
    const uint32_t b0 = min((uint32_t)(x0 / unit), nb), b1 = min((uint32_t)((x0 + kStripCols) / unit), nb);
    if (b1 > b0) {
      const EdgeSeg *g = a.grid[plane] + (size_t)b0 * a.grid_slots[plane];
      if (plane == 0) run_cell_runs<4, kStripCols>(a, view, g, a.grid_slots[plane], b1 - b0);
      else run_cell_runs<2, kStripCols>(a, view, g, a.grid_slots[plane], b1 - b0);
    }
  } else {
    const uint32_t *bf = a.band_first + a.band_off[plane];
    const uint32_t nb = a.n_bands[plane];
    const uint32_t b0 = min((uint32_t)(x0 / unit), nb), b1 = min((uint32_t)((x0 + kStripCols) / unit), nb);
    if (plane == 0) run_components<4, kStripCols>(a, view, bf[b0], bf[b1]);
    else run_components<2, kStripCols>(a, view, bf[b0], bf[b1]);
  }
  __syncthreads();
  if (vec) {
    for (int i = threadIdx.x; i < h * kStripVec; i += blockDim.x) {
      const int r = i / kStripVec, c = (i % kStripVec) * 8;
      *reinterpret_cast<uint4 *>(p.s + (int64_t)r * p.stride + x0 + c) =
          *reinterpret_cast<const uint4 *>(sm + r * kStripCols + c);
    }
  } else {
    for (int i = threadIdx.x; i < h * cols; i += blockDim.x) {
      const int r = i / cols, c = i - r * cols;
      p.s[(int64_t)r * p.stride + x0 + c] = sm[r * kStripCols + c];
    }
  }
}

// ------------------------------------------------------------ tile kernel
// One CTA per 64x64 luma tile and its 32x32 chroma tiles.  The tile's region
// -- the tile widened by the halo -- is staged once by TMA box loads (luma
// then through the LMCS LUT in shared memory) while the tile's components are
// staged in shared memory; the vertical-pass components that reach the
// tile's columns in the widened rows run, then the horizontal-pass components
// that reach the tile, and the tile itself is stored.  A component that two
// tiles need runs in both on the same samples, so no CTA reads another's
// output.  Components span at most the halo (checked on the host, or by
// construction for the device walk's pictures), so every clamped read of a
// listed component stays inside the region.
constexpr int kTileThreads = 256;
constexpr int kRegionY = kDeblockTile + 2 * kDeblockHaloY;      // 96
constexpr int kRegionC = kDeblockTile / 2 + 2 * kDeblockHaloC;  // 48
constexpr int kPitchY = kRegionY + 8;                           // smem row pitch, samples
constexpr int kPitchC = kRegionC + 8;
constexpr size_t kTileSmem = (size_t)(kRegionY * kPitchY + 2 * kRegionC * kPitchC) * 2;

struct TileParams {
  DPlane src[3], dst[3];
  const EdgeSeg *segs[2];
  const uint32_t *comp[2];
  const uint32_t *bounds;  // component ranges per (band, tile), see DeblockPlan::tile_bounds
  uint32_t tb_off[2][3];
  uint32_t n_bands[2][3];
  const uint16_t *lut;
  uint32_t tiles_x, tiles_y;
  int maxv;
  // Grid mode (side information built on the device): every component is one
  // segment, stored in grid[d][p][band * grid_slots[d][p] + pos / unit] (bs 0:
  // none), unit 4 luma / 8 chroma samples along the edge normal; the walk
  // lists each tile's cells.
  int grid_mode;
  const EdgeSeg *grid[2][3];
  uint32_t grid_slots[2][3];
  const uint32_t *grid_count;       // cells per (tile, pass, plane), listed by the walk
  const uint32_t *grid_list[2][3];  // their grid indices, kTileListY / kTileListC per tile
  // The regions staged by the TMA unit: one box per plane, kPitch wide and
  // kRegion high, at the tile's origin less the halo (tma 0: vector loads).
  int tma;
  CUtensorMap tmap[3];
};

constexpr int kTileBands = 32;

// Tiles whose region copies did not complete within the poll limit (left
// unwritten); read and cleared by deblock_wait_timeouts.
__device__ unsigned int g_deblock_timeouts;  // bands of one tile and pass that a plane can have (at most 24)

// Copies rows [oy, oy + wh) x columns [ox, ox + ww) of `src` (ox a multiple of
// 8) to shared memory with row pitch `pitch`, mapping through `lut` if given.
__device__ __forceinline__ void load_window(uint16_t *sm, int pitch, const DPlane &src, int ox, int oy, int ww,
                                            int wh, const uint16_t *lut) {
  const int nvec = vec_ok(src) ? ww / 8 : 0, tail = ww - nvec * 8;
  for (int i = threadIdx.x; i < wh * nvec; i += blockDim.x) {
    const int r = i / nvec, c = (i - r * nvec) * 8;
    uint4 q = *reinterpret_cast<const uint4 *>(src.s + (int64_t)(oy + r) * src.stride + ox + c);
    if (lut) {
      uint32_t *u = reinterpret_cast<uint32_t *>(&q);
#pragma unroll
      for (int k = 0; k < 4; ++k) u[k] = (uint32_t)lut[u[k] & 0xFFFF] | (uint32_t)lut[u[k] >> 16] << 16;
    }
    *reinterpret_cast<uint4 *>(sm + r * pitch + c) = q;
  }
  for (int i = threadIdx.x; i < wh * tail; i += blockDim.x) {
    const int r = i / tail, c = nvec * 8 + (i - r * tail);
    const uint16_t x = src.s[(int64_t)(oy + r) * src.stride + ox + c];
    sm[r * pitch + c] = lut ? lut[x] : x;
  }
}

// Stores rows [y0, y0 + ih) x columns [x0, x0 + iw) (x0 a multiple of 8) from
// the window whose origin is (ox, oy).
__device__ __forceinline__ void store_window(const uint16_t *sm, int pitch, const DPlane &dst, int ox, int oy,
                                             int x0, int y0, int iw, int ih) {
  const int nvec = vec_ok(dst) ? iw / 8 : 0, tail = iw - nvec * 8;
  const uint16_t *s0 = sm + (y0 - oy) * pitch + (x0 - ox);
  for (int i = threadIdx.x; i < ih * nvec; i += blockDim.x) {
    const int r = i / nvec, c = (i - r * nvec) * 8;
    *reinterpret_cast<uint4 *>(dst.s + (int64_t)(y0 + r) * dst.stride + x0 + c) =
        *reinterpret_cast<const uint4 *>(s0 + r * pitch + c);
  }
  for (int i = threadIdx.x; i < ih * tail; i += blockDim.x) {
    const int r = i / tail, c = nvec * 8 + (i - r * tail);
    dst.s[(int64_t)(y0 + r) * dst.stride + x0 + c] = s0[r * pitch + c];
  }
}

// Band counts and prefix sums of the tile's component ranges for (pass d,
// plane p), by one warp.
// The staged window of plane p of tile (tx, ty): the tile widened by the
// halo, clipped to the plane.  Recomputed where needed rather than kept live.
__device__ __forceinline__ SharedView tile_view(const TileParams &a, uint16_t *sm, int p, int tx, int ty) {
  const DPlane &src = a.src[p];
  const int tp = p ? kDeblockTile / 2 : kDeblockTile, halo = p ? kDeblockHaloC : kDeblockHaloY;
  const int pitch = p ? kPitchC : kPitchY;
  uint16_t *box = p == 0 ? sm : sm + kRegionY * kPitchY + (p - 1) * kRegionC * kPitchC;
  const int rx = tx * tp - halo, ry = ty * tp - halo;  // the box's origin, before clipping to the plane
  const int ox = max(rx, 0), oy = max(ry, 0);
  const int ww = min(tx * tp + tp + halo, src.w) - ox, wh = min(ty * tp + tp + halo, src.h) - oy;
  return SharedView{box + (oy - ry) * pitch + (ox - rx), pitch, ox, oy, max(ww, 0), max(wh, 0), src.w, src.h};
}

// An EdgeSeg moved as three 32-bit words (every array of them here starts on
// a 4-byte boundary: blob sections, grid cells and shared arrays).
union SegWords {
  EdgeSeg e;
  uint32_t w[3];
};
__device__ __forceinline__ EdgeSeg seg_get(const EdgeSeg *p) {
  const uint32_t *w = reinterpret_cast<const uint32_t *>(p);
  SegWords u;
  u.w[0] = w[0];
  u.w[1] = w[1];
  u.w[2] = w[2];
  return u.e;
}
__device__ __forceinline__ void seg_copy(EdgeSeg *dst, const EdgeSeg *src) {
  const uint32_t *s = reinterpret_cast<const uint32_t *>(src);
  uint32_t *d = reinterpret_cast<uint32_t *>(dst);
  const uint32_t a = s[0], b = s[1], c = s[2];
  d[0] = a;
  d[1] = b;
  d[2] = c;
}

// The tile's components of one (pass, plane), staged in shared memory before
// the filters run: their segments one component after another and each
// component's first segment (start[n] ends the last one), so the filter
// phase reads no global memory.
struct TileStage {
  EdgeSeg *seg;
  uint16_t *start;
  uint32_t cap;
};

// The largest b in [0, 31] with prefix[b] <= x (prefix non-decreasing,
// prefix[0] = 0): the band holding entry x.
__device__ __forceinline__ int band_of(const uint32_t *prefix, uint32_t x) {
  int b = 0;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1)
    if (prefix[b + s] <= x) b += s;
  return b;
}

// Host-built lists, by one warp: lane b reads the component range of band
// b0 + b of the tile, the prefix sums over the lanes give each band's first
// component and segment in the staged arrays, then the warp stages every
// component start and segment.  `band` is the warp's scratch (4 x 33).  The
// host keeps every tile's segment count within the caps.
__device__ __forceinline__ uint32_t stage_host(const TileParams &a, int d, int p, int tx, int ty, const TileStage &st,
                                               uint32_t (*band)[kTileBands + 1]) {
  const int lane = threadIdx.x & 31;
  const int tp = p ? kDeblockTile / 2 : kDeblockTile, halo = p ? kDeblockHaloC : kDeblockHaloY, unit = p ? 2 : 4;
  const int nb = (int)a.n_bands[d][p];
  int b0, b1, n_t, t;
  if (d == 0) {  // row bands of the tile's rows widened by the halo
    b0 = max(ty * tp - halo, 0) / unit;
    b1 = min((ty * tp + tp + halo) / unit, nb);
    n_t = (int)a.tiles_x;
    t = tx;
  } else {  // column bands of the tile
    b0 = tx * tp / unit;
    b1 = min((tx * tp + tp) / unit, nb);
    n_t = (int)a.tiles_y;
    t = ty;
  }
  const uint32_t *comp = a.comp[d];
  const int b = b0 + lane;
  uint32_t lo = 0, cnt = 0, s0 = 0, ns = 0;
  if (b < b1) {
    const uint32_t *e = a.bounds + a.tb_off[d][p] + ((size_t)b * n_t + t) * 2;
    lo = e[0];
    cnt = e[1] - e[0];
    if (cnt) {
      s0 = comp[lo];
      ns = comp[lo + cnt] - s0;
    }
  }
  uint32_t ic = cnt, is = ns;  // inclusive prefix sums over the lanes
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t yc = __shfl_up_sync(0xFFFFFFFFu, ic, o), ys = __shfl_up_sync(0xFFFFFFFFu, is, o);
    if (lane >= o) {
      ic += yc;
      is += ys;
    }
  }
  band[0][lane] = ic - cnt;
  band[1][lane] = is - ns;
  band[2][lane] = lo;
  band[3][lane] = s0;
  const uint32_t nc = min(__shfl_sync(0xFFFFFFFFu, ic, 31), st.cap), nseg = min(__shfl_sync(0xFFFFFFFFu, is, 31), st.cap);
  __syncwarp();
  for (uint32_t j = lane; j < nc; j += 32) {
    const int k = band_of(band[0], j);
    const uint32_t c = band[2][k] + j - band[0][k];
    st.start[j] = (uint16_t)min(band[1][k] + comp[c] - band[3][k], nseg);
  }
  if (lane == 0) st.start[nc] = (uint16_t)nseg;
  const EdgeSeg *segs = a.segs[d];
  for (uint32_t i = lane; i < nseg; i += 32) {
    const int k = band_of(band[1], i);
    seg_copy(st.seg + i, segs + band[3][k] + i - band[1][k]);
  }
  return nc;
}

// Grid mode, by one warp: the cells the device walk listed for (pass d,
// plane p) of tile t, each its own component.
__device__ __forceinline__ uint32_t stage_grid(const TileParams &a, int d, int p, int t, const TileStage &st) {
  const int lane = threadIdx.x & 31;
  const uint32_t n = min(a.grid_count[(size_t)t * 6 + d * 3 + p], st.cap);
  const uint32_t *src = a.grid_list[d][p] + (size_t)t * st.cap;
  const EdgeSeg *g = a.grid[d][p];
  for (uint32_t j = lane; j < n; j += 32) {
    seg_copy(st.seg + j, g + src[j]);
    st.start[j] = (uint16_t)j;
  }
  if (lane == 0) st.start[n] = (uint16_t)n;
  return n;
}

struct TileShared {
  alignas(16) EdgeSeg seg_y[2][kTileListY];
  alignas(16) EdgeSeg seg_c[2][2][kTileListC];
  uint16_t start_y[2][kTileListY + 1], start_c[2][2][kTileListC + 1];
  uint32_t band[6][4][kTileBands + 1];  // stage_host scratch per (pass, plane)
  uint32_t n_comp[2][3];
  uint32_t task[2];                   // the passes' next warp task
  alignas(8) unsigned long long bar;  // completion of the TMA region copies
  __device__ TileStage stage(int d, int p) {
    return p == 0 ? TileStage{seg_y[d], start_y[d], (uint32_t)kTileListY}
                  : TileStage{seg_c[d][p - 1], start_c[d][p - 1], (uint32_t)kTileListC};
  }
};

// The components of one pass of a tile, all three planes, spread over the
// CTA's warps: a warp task is 8 luma components (groups of 4 lanes) or 16
// chroma components (groups of 2), so no plane waits for another; warps take
// tasks from a shared counter, so a warp with long components does not hold
// the others at the pass's barrier.
__device__ __forceinline__ void run_tile_pass(const TileParams &a, uint16_t *sm, TileShared &ts, int tx, int ty,
                                              int d) {
  const int lane = threadIdx.x & 31;
  const uint32_t n0 = ts.n_comp[d][0], n1 = ts.n_comp[d][1], n2 = ts.n_comp[d][2];
  const uint32_t tasks0 = (n0 + 7) / 8, tasks1 = (n1 + 15) / 16, tasks2 = (n2 + 15) / 16;
  const uint32_t total = tasks0 + tasks1 + tasks2;
  for (;;) {
    uint32_t t = 0;
    if (lane == 0) t = atomicAdd(&ts.task[d], 1u);
    t = __shfl_sync(0xFFFFFFFFu, t, 0);
    if (t >= total) break;
    if (t < tasks0) {
      const int k = lane & 3, base = lane - k;
      const unsigned mask = 0xFu << base;
      const uint32_t j = t * 8 + (lane >> 2);
      if (j < n0) {
        const SharedView v = tile_view(a, sm, 0, tx, ty);
        const uint32_t e = ts.start_y[d][j + 1];
        for (uint32_t i = ts.start_y[d][j]; i < e; ++i) {
          segment_group<4, kPitchY>(v, seg_get(&ts.seg_y[d][i]), a.maxv, k, base, mask);
          __syncwarp(mask);
        }
      }
    } else {
      const bool cr = t >= tasks0 + tasks1;
      const int c = cr ? 1 : 0;
      const uint32_t tt = t - tasks0 - (cr ? tasks1 : 0);
      const int k = lane & 1, base = lane - k;
      const unsigned mask = 0x3u << base;
      const uint32_t j = tt * 16 + (lane >> 1);
      if (j < (cr ? n2 : n1)) {
        const SharedView v = tile_view(a, sm, cr ? 2 : 1, tx, ty);
        const uint32_t e = ts.start_c[d][c][j + 1];
        for (uint32_t i = ts.start_c[d][c][j]; i < e; ++i) {
          segment_group<2, kPitchC>(v, seg_get(&ts.seg_c[d][c][i]), a.maxv, k, base, mask);
          __syncwarp(mask);
        }
      }
    }
  }
}

// Tile t of the picture whose parameters are `a` (`g`: the same parameters in
// global or parameter memory, for the tensor maps).
__device__ __forceinline__ void deblock_tile(const TileParams &a, const TileParams *g, int t) {
  extern __shared__ __align__(128) uint16_t sm_tile[];  // TMA destinations: 128-byte aligned
  uint16_t *sm = sm_tile;
  __shared__ TileShared ts;
  const int tx = t % (int)a.tiles_x, ty = t / (int)a.tiles_x;
  const int warp = threadIdx.x >> 5;
  // Thread 0 starts the TMA copies of the planes' regions; meanwhile warps
  // 0-5 stage the components of both passes (one warp per pass and plane,
  // from the host's ranges or the device walk's lists).
  if (threadIdx.x == 0) {
    ts.task[0] = ts.task[1] = 0;
    if (a.tma) {
      tile_dev::mbar_init(&ts.bar, 1);
      uint32_t bytes = 0;
#pragma unroll
      for (int p = 0; p < 3; ++p)
        if (a.src[p].w > 0 && a.src[p].h > 0) bytes += (p ? kRegionC * kPitchC : kRegionY * kPitchY) * 2;
      tile_dev::mbar_expect_tx(&ts.bar, bytes);
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        if (a.src[p].w <= 0 || a.src[p].h <= 0) continue;
        const int tp = p ? kDeblockTile / 2 : kDeblockTile, halo = p ? kDeblockHaloC : kDeblockHaloY;
        uint16_t *box = p == 0 ? sm : sm + kRegionY * kPitchY + (p - 1) * kRegionC * kPitchC;
        tile_dev::tmap_acquire(&g->tmap[p]);
        tile_dev::tma_load_2d(box, &g->tmap[p], tx * tp - halo, ty * tp - halo, &ts.bar);
      }
    }
  }
  if (warp < 6) {
    const int d = warp / 3, p = warp % 3;
    const uint32_t n = a.grid_mode ? stage_grid(a, d, p, t, ts.stage(d, p))
                                   : stage_host(a, d, p, tx, ty, ts.stage(d, p), ts.band[warp]);
    if ((threadIdx.x & 31) == 0) ts.n_comp[d][p] = n;
  }
  if (!a.tma) {
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      const SharedView v = tile_view(a, sm, p, tx, ty);
      if (v.ww > 0 && v.wh > 0) load_window(v.s, v.ld, a.src[p], v.ox, v.oy, v.ww, v.wh, p == 0 ? a.lut : nullptr);
    }
    __syncthreads();
  } else {
    __syncthreads();  // the barrier's initialisation and the staged components
    bool ok = tile_dev::mbar_wait_bounded(&ts.bar, 0);
    if (ok && a.lut) {  // luma through the LMCS LUT, in place (the whole box: samples outside the plane are never read)
      uint32_t *w = reinterpret_cast<uint32_t *>(sm);
      for (int i = threadIdx.x; i < kRegionY * kPitchY / 2; i += blockDim.x) {
        const uint32_t u = w[i];
        w[i] = (uint32_t)a.lut[u & 0xFFFF] | (uint32_t)a.lut[u >> 16] << 16;
      }
    }
    ok = __syncthreads_and(ok);
    if (!ok) {  // the copies did not land in time: count it, let them finish (bounded), leave the tile
      if (threadIdx.x == 0) {
        atomicAdd(&g_deblock_timeouts, 1u);
        tile_dev::mbar_wait_bounded(&ts.bar, 0);
      }
      return;
    }
  }
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    run_tile_pass(a, sm, ts, tx, ty, d);
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    const SharedView v = tile_view(a, sm, p, tx, ty);
    const int tp = p ? kDeblockTile / 2 : kDeblockTile, x0 = tx * tp, y0 = ty * tp;
    const int iw = min(x0 + tp, a.dst[p].w) - x0, ih = min(y0 + tp, a.dst[p].h) - y0;
    if (iw > 0 && ih > 0 && v.ww > 0 && v.wh > 0) store_window(v.s, v.ld, a.dst[p], v.ox, v.oy, x0, y0, iw, ih);
  }
}

__global__ void __launch_bounds__(kTileThreads, 4) k_deblock_tiles(const __grid_constant__ TileParams a) {
  deblock_tile(a, &a, blockIdx.x);
}

// Many pictures in one grid: CTAs [first[i], first[i + 1]) are the tiles of
// picture i, whose parameters are params[i].
__global__ void __launch_bounds__(kTileThreads, 4) k_deblock_tiles_batch(const TileParams *__restrict__ params,
                                                                         const uint32_t *__restrict__ first, int n) {
  __shared__ TileParams s_params;  // the picture's parameters, read once per CTA
  int lo = 0, hi = n;               // first[lo] <= blockIdx.x < first[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (first[mid] <= blockIdx.x) lo = mid;
    else hi = mid;
  }
  static_assert(sizeof(TileParams) % 4 == 0, "word copy");
  const uint32_t *src = reinterpret_cast<const uint32_t *>(params + lo);
  uint32_t *dst = reinterpret_cast<uint32_t *>(&s_params);
  for (int i = threadIdx.x; i < (int)(sizeof(TileParams) / 4); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  deblock_tile(s_params, params + lo, (int)(blockIdx.x - first[lo]));
}

size_t rows_smem(const DPlane &p) { return (size_t)4 * row_pitch(p.w) * 2; }
size_t cols_smem(const DPlane &p) { return (size_t)p.h * kStripCols * 2; }

}  // namespace

bool deblock_strips_fit(const DPlane planes[3]) {
  for (int i = 0; i < 3; ++i) {
    if ((int64_t)planes[i].w * planes[i].h == 0) continue;
    if (rows_smem(planes[i]) > (size_t)kMaxStripSmem || cols_smem(planes[i]) > (size_t)kMaxStripSmem) return false;
  }
  return true;
}

int launch_deblock_strips(cudaStream_t st, const DPlane src[3], const DPlane dst[3], const uint16_t *lut,
                          int bit_depth, const StripSide &v, const StripSide &h, const uint32_t band_off[2][3],
                          const uint32_t n_bands[2][3], uint64_t *launches) {
  StripParams a;
  std::memset(&a, 0, sizeof a);
  size_t smem_rows = 0, smem_cols = 0;
  uint32_t ctas_rows = 0, ctas_cols = 0;
  uint32_t strips[3];
  for (int i = 0; i < 3; ++i) {
    a.src[i] = src[i];
    a.dst[i] = dst[i];
    const bool empty = (int64_t)src[i].w * src[i].h == 0;
    strips[i] = empty ? 0 : (uint32_t)((src[i].w + kStripCols - 1) / kStripCols);
    if (!empty) {
      smem_rows = std::max(smem_rows, rows_smem(src[i]));
      smem_cols = std::max(smem_cols, cols_smem(src[i]));
    }
    ctas_rows += empty ? 0 : n_bands[0][i];
    ctas_cols += strips[i];
  }
  a.lut = lut;
  a.maxv = (1 << bit_depth) - 1;
  // vertical pass
  a.segs = v.segs;
  a.comp = v.comp;
  a.band_first = v.band_first;
  for (int i = 0; i < 3; ++i) {
    a.band_off[i] = band_off[0][i];
    a.n_bands[i] = n_bands[0][i];
    a.ctas[i] = (int64_t)src[i].w * src[i].h ? n_bands[0][i] : 0;
  }
  if (ctas_rows) {
    if (smem_rows > 48 * 1024)
      H266_CUDA(cudaFuncSetAttribute(k_deblock_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_rows));
    k_deblock_rows<<<ctas_rows, 128, smem_rows, st>>>(a);
    H266_CUDA(cudaGetLastError());
    ++*launches;
  }
  // horizontal pass, in place on dst
  a.segs = h.segs;
  a.comp = h.comp;
  a.band_first = h.band_first;
  a.lut = nullptr;
  for (int i = 0; i < 3; ++i) {
    a.band_off[i] = band_off[1][i];
    a.n_bands[i] = n_bands[1][i];
    a.ctas[i] = strips[i];
  }
  if (ctas_cols) {
    if (smem_cols > 48 * 1024)
      H266_CUDA(cudaFuncSetAttribute(k_deblock_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cols));
    k_deblock_cols<<<ctas_cols, 128, smem_cols, st>>>(a);
    H266_CUDA(cudaGetLastError());
    ++*launches;
  }
  return H266_OK;
}

// Strip kernels on the device walk's cell grids: a CTA per row band of each
// plane (vertical pass, src -> dst), then per 8-column strip (horizontal pass,
// in place on dst).  Row bands follow the plane sizes, so planes without
// segments (chroma of a 4:0:0 walk) are still copied.
int launch_deblock_strips_grid(cudaStream_t st, const DPlane src[3], const DPlane dst[3], const uint16_t *lut,
                               int bit_depth, const DeviceWalkOut &g, uint64_t *launches) {
  StripParams a;
  std::memset(&a, 0, sizeof a);
  a.grid_mode = 1;
  size_t smem_rows = 0, smem_cols = 0;
  uint32_t ctas_rows = 0, ctas_cols = 0, rows[3], strips[3];
  for (int i = 0; i < 3; ++i) {
    a.src[i] = src[i];
    a.dst[i] = dst[i];
    const bool empty = (int64_t)src[i].w * src[i].h == 0;
    const int unit = i ? 2 : 4;
    rows[i] = empty ? 0 : (uint32_t)((src[i].h + unit - 1) / unit);
    strips[i] = empty ? 0 : (uint32_t)((src[i].w + kStripCols - 1) / kStripCols);
    if (!empty) {
      smem_rows = std::max(smem_rows, rows_smem(src[i]));
      smem_cols = std::max(smem_cols, cols_smem(src[i]));
    }
    ctas_rows += rows[i];
    ctas_cols += strips[i];
  }
  if (smem_rows > (size_t)kMaxStripSmem || smem_cols > (size_t)kMaxStripSmem)
    return set_error(H266_ERR_UNSUPPORTED, "deblock: planes too large for the strip kernels");
  a.lut = lut;
  a.maxv = (1 << bit_depth) - 1;
  for (int i = 0; i < 3; ++i) {
    a.grid[i] = g.grid[0][i];
    a.grid_slots[i] = g.slots[0][i];
    a.grid_bands[i] = g.bands[0][i];
    a.ctas[i] = rows[i];
  }
  if (ctas_rows) {
    if (smem_rows > 48 * 1024)
      H266_CUDA(cudaFuncSetAttribute(k_deblock_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_rows));
    k_deblock_rows<<<ctas_rows, 128, smem_rows, st>>>(a);
    H266_CUDA(cudaGetLastError());
    ++*launches;
  }
  a.lut = nullptr;
  for (int i = 0; i < 3; ++i) {
    a.grid[i] = g.grid[1][i];
    a.grid_slots[i] = g.slots[1][i];
    a.grid_bands[i] = g.bands[1][i];
    a.ctas[i] = strips[i];
  }
  if (ctas_cols) {
    if (smem_cols > 48 * 1024)
      H266_CUDA(cudaFuncSetAttribute(k_deblock_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cols));
    k_deblock_cols<<<ctas_cols, 128, smem_cols, st>>>(a);
    H266_CUDA(cudaGetLastError());
    ++*launches;
  }
  return H266_OK;
}

size_t deblock_tile_params_size() { return sizeof(TileParams); }

namespace {
// The tile kernels' shared memory (staged components, parameters and the
// regions, above the 48 KB default) and a full carveout, once per device.
int prepare_tile_kernels() {
  static std::atomic<uint64_t> done{0};
  int dev = 0;
  H266_CUDA(cudaGetDevice(&dev));
  const uint64_t bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_relaxed) & bit) return H266_OK;
  for (const void *k : {reinterpret_cast<const void *>(k_deblock_tiles), reinterpret_cast<const void *>(k_deblock_tiles_batch)}) {
    H266_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmem));
    H266_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  }
  done.fetch_or(bit);
  return H266_OK;
}
}  // namespace

int deblock_wait_timeouts(uint32_t *count) {
  unsigned int v = 0, zero = 0;
  H266_CUDA(cudaMemcpyFromSymbol(&v, g_deblock_timeouts, sizeof v));
  if (v) H266_CUDA(cudaMemcpyToSymbol(g_deblock_timeouts, &zero, sizeof zero));
  *count = v;
  return H266_OK;
}

namespace {
// The tensor maps of the tile kernel's region boxes (a.tma 0 when a plane
// cannot be described: unaligned base or stride).
void tile_tma_maps(TileParams &a) {
  bool ok = true;
  for (int p = 0; p < 3 && ok; ++p)
    if (a.src[p].w > 0 && a.src[p].h > 0)
      ok = encode_plane_map(&a.tmap[p], a.src[p], p ? kPitchC : kPitchY, p ? kRegionC : kRegionY);
  a.tma = ok ? 1 : 0;
}
}  // namespace

uint32_t fill_deblock_tile_params(void *out, const DPlane src[3], const DPlane dst[3], const uint16_t *lut,
                                  int bit_depth, const StripSide &v, const StripSide &h, const uint32_t *tile_bounds,
                                  const uint32_t tb_off[2][3], const uint32_t n_bands[2][3], uint32_t tiles_x,
                                  uint32_t tiles_y) {
  TileParams a;
  std::memset(&a, 0, sizeof a);
  for (int i = 0; i < 3; ++i) {
    a.src[i] = src[i];
    a.dst[i] = dst[i];
    for (int d = 0; d < 2; ++d) {
      a.tb_off[d][i] = tb_off[d][i];
      a.n_bands[d][i] = n_bands[d][i];
    }
  }
  a.segs[0] = v.segs;
  a.comp[0] = v.comp;
  a.segs[1] = h.segs;
  a.comp[1] = h.comp;
  a.bounds = tile_bounds;
  a.lut = lut;
  a.tiles_x = tiles_x;
  a.tiles_y = tiles_y;
  a.maxv = (1 << bit_depth) - 1;
  tile_tma_maps(a);
  std::memcpy(out, &a, sizeof a);
  return tiles_x * tiles_y;
}

int launch_deblock_tiles(cudaStream_t st, const DPlane src[3], const DPlane dst[3], const uint16_t *lut,
                         int bit_depth, const StripSide &v, const StripSide &h, const uint32_t *tile_bounds,
                         const uint32_t tb_off[2][3], const uint32_t n_bands[2][3], uint32_t tiles_x,
                         uint32_t tiles_y, uint64_t *launches) {
  TileParams a;
  const uint32_t n = fill_deblock_tile_params(&a, src, dst, lut, bit_depth, v, h, tile_bounds, tb_off, n_bands,
                                              tiles_x, tiles_y);
  if (!n) return H266_OK;
  H266_TRY(prepare_tile_kernels());
  k_deblock_tiles<<<n, kTileThreads, kTileSmem, st>>>(a);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

int launch_deblock_tiles_batch(cudaStream_t st, const void *d_params, const uint32_t *d_first, int n, uint32_t ctas,
                               uint64_t *launches) {
  if (!ctas || n <= 0) return H266_OK;
  H266_TRY(prepare_tile_kernels());
  k_deblock_tiles_batch<<<ctas, kTileThreads, kTileSmem, st>>>(static_cast<const TileParams *>(d_params), d_first, n);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

int launch_deblock(cudaStream_t st, const DPlane planes[3], int bit_depth, const EdgeSeg *d_segs_v,
                   const uint32_t *d_comp_v, uint32_t n_comp_v, const EdgeSeg *d_segs_h, const uint32_t *d_comp_h,
                   uint32_t n_comp_h, uint64_t *launches) {
  Planes3 p3{{planes[0], planes[1], planes[2]}};
  const int maxv = (1 << bit_depth) - 1;
  if (n_comp_v) {
    k_deblock_components<<<(n_comp_v + 127) / 128, 128, 0, st>>>(p3, d_segs_v, d_comp_v, n_comp_v, maxv);
    H266_CUDA(cudaGetLastError());
    ++*launches;
  }
  if (n_comp_h) {
    k_deblock_components<<<(n_comp_h + 127) / 128, 128, 0, st>>>(p3, d_segs_h, d_comp_h, n_comp_h, maxv);
    H266_CUDA(cudaGetLastError());
    ++*launches;
  }
  return H266_OK;
}

// ===================================================================== device-built side information
int device_walk_mode(const h266_picture &pic, const h266_deblock_cu *cus, uint64_t n_cus,
                     const h266_deblock_cu *chroma_cus, uint64_t n_chroma, const h266_deblock_params &params,
                     uint32_t cfi) {
  if (params.disabled || params.bit_depth < 8 || params.bit_depth > 16 || params.ctb_log2_size_y > 16) return 0;
  if (cfi > 3) return 0;
  const int w = (int)pic.luma.width, h = (int)pic.luma.height;
  if (w <= 0 || h <= 0) return 0;
  const bool chroma = (uint64_t)pic.cb.width * pic.cb.height != 0 || (uint64_t)pic.cr.width * pic.cr.height != 0;
  if (n_cus > (uint64_t)INT32_MAX || n_chroma > (uint64_t)INT32_MAX) return 0;
  // The tile kernel's condition: no two segments' footprints overlap, every
  // one inside a cell of the tile halo -- luma CUs and transform blocks at
  // least 8 samples, no sub-block edges, 4:2:0 or 4:0:0.
  bool no_chains = cfi <= 1 && !(cfi == 0 && chroma);
  if (chroma && (pic.cb.width != (pic.luma.width + 1) / 2 || pic.cb.height != (pic.luma.height + 1) / 2 ||
                 pic.cr.width != pic.cb.width || pic.cr.height != pic.cb.height))
    no_chains = false;
  // The strip kernels' condition: a plane's row band and full-height strip fit
  // their shared memory.
  const h266_plane *pl[3] = {&pic.luma, &pic.cb, &pic.cr};
  for (int i = 0; i < 3; ++i) {
    const DPlane d{nullptr, 0, (int)pl[i]->width, (int)pl[i]->height};
    if ((int64_t)d.w * d.h && (rows_smem(d) > (size_t)kMaxStripSmem || cols_smem(d) > (size_t)kMaxStripSmem))
      return 0;
  }
  // CUs on the 4x4 grid, inside the picture, not overlapping (the walk's
  // emissions then never share a grid cell), and in decode order along every
  // row and column of the CU map: then a band's segments come out of the
  // reference's walk in position order, the order the strip kernels run a
  // chain of overlapping footprints in.
  const int cw4 = (w + 3) / 4, ch4 = (h + 3) / 4, words = (cw4 + 63) / 64;
  thread_local std::vector<uint64_t> bits;  // occupied 4x4 cells, one bit each
  thread_local std::vector<int32_t> map, last_col;
  const h266_deblock_cu *lists[2] = {cus, chroma_cus};
  const uint64_t counts[2] = {n_cus, chroma_cus ? n_chroma : 0};
  for (int l = 0; l < 2; ++l) {
    if (!lists[l]) continue;
    bits.assign((size_t)words * ch4, 0);
    bool chains = false;  // 4-sample edges, sub-block edges or narrow transform blocks in this list
    for (uint64_t i = 0; i < counts[l]; ++i) {
      const h266_deblock_cu &c = lists[l][i];
      if ((c.x | c.y | c.w | c.h) & 3 || c.w == 0 || c.h == 0) return 0;
      if ((uint64_t)c.x + c.w > (uint64_t)w || (uint64_t)c.y + c.h > (uint64_t)h) return 0;
      if (c.has_tb_split && (c.tb_split.n_bounds < 1 || c.tb_split.n_bounds > 3)) return 0;
      if (c.w < 8 || c.h < 8 || c.has_num_sb) chains = true;
      if (c.has_tb_split) {
        const uint32_t dim = c.tb_split.vertical ? c.w : c.h;
        uint32_t prev = 0;
        for (int k = 0; k < c.tb_split.n_bounds; ++k) {
          const uint32_t b = c.tb_split.bounds[k];
          if (b < prev + 8) chains = true;
          prev = b;
        }
        if (dim < prev + 8) chains = true;
      }
      const uint32_t x0 = c.x / 4, x1 = (c.x + c.w) / 4;
      for (uint32_t y = c.y / 4; y < (c.y + c.h) / 4; ++y) {
        uint64_t *row = bits.data() + (size_t)y * words;
        for (uint32_t x = x0; x < x1;) {  // the run's part inside one 64-cell word
          const uint32_t wi = x / 64, lo = x % 64, n = std::min<uint32_t>(x1 - x, 64 - lo);
          const uint64_t m = (n == 64 ? ~0ull : ((1ull << n) - 1)) << lo;
          if (row[wi] & m) return 0;  // overlaps an earlier CU
          row[wi] |= m;
          x += n;
        }
      }
    }
    if (chains) no_chains = false;
    // Only luma footprints chain (chroma edges are 8 chroma samples apart and
    // reach 4), so only the luma list's order matters.
    if (l != 0 || !chains) continue;
    map.assign((size_t)cw4 * ch4, -1);
    for (uint64_t i = 0; i < counts[l]; ++i) {
      const h266_deblock_cu &c = lists[l][i];
      for (uint32_t y = c.y / 4; y < (c.y + c.h) / 4; ++y)
        std::fill(map.begin() + (size_t)y * cw4 + c.x / 4, map.begin() + (size_t)y * cw4 + (c.x + c.w) / 4,
                  (int32_t)i);
    }
    last_col.assign((size_t)cw4, -1);
    for (int y = 0; y < ch4; ++y) {
      int32_t last_row = -1;
      const int32_t *row = map.data() + (size_t)y * cw4;
      for (int x = 0; x < cw4; ++x) {
        const int32_t v = row[x];
        if (v < 0) continue;
        if (v < last_row || v < last_col[x]) return 0;
        last_row = v;
        last_col[x] = v;
      }
    }
  }
  return no_chains ? 1 : 2;
}

namespace {

struct DevCuGrid {  // CuGrid::cu_at on device memory
  const int32_t *cells;
  int cw, ch;
  __device__ int64_t at(int x, int y) const {
    if (x < 0 || y < 0 || x / 4 >= cw || y / 4 >= ch) return -1;
    return cells[(size_t)(y / 4) * cw + x / 4];
  }
};

// Motion by CU: every 4x4 cell of a CU carries the same motion (checked on
// the host), so the cell's motion is its CU's record.
struct CuMotion {
  const h266_deblock_mv_grid *g;  // presence only
  const h266_deblock_mv_cell *per_cu;
  DevCuGrid grid;
  __device__ const h266_deblock_mv_cell &at(int x, int y) const {
    const int64_t i = grid.at(x, y);
    return i < 0 ? kNoMotionDev : per_cu[i];
  }
};

struct WalkParams {
  h266_deblock_cu *cus[2];  // luma list, chroma list: full records, expanded in the walk's scratch
  uint32_t n[2];
  const uint8_t *heads[2];  // the staged packed lists (see CuCompact, CuTail, CuMotionRec)
  int compact[2];
  const CuTail *tails[2];
  uint32_t n_tails[2];
  const CuMotionRec *mv_recs;
  uint32_t n_mv_recs;
  int32_t *cu_grid[2];
  int cw4, ch4;
  h266_deblock_mv_grid mv;
  int has_mv;
  h266_deblock_mv_cell *mv_per_cu;  // non-null: motion by luma CU instead of the grid (expanded)
  const uint32_t *nf[2];  // columns (vertical pass), rows (horizontal pass)
  uint32_t n_nf[2];
  PlaneCfg cfg[3];
  EdgeSeg *grid[2][3];
  uint32_t slots[2][3], bands[2][3];
  // Per-tile lists for the grid-mode tile kernel (null when the strip kernels
  // consume the grids): tile_count[tile * 6 + pass * 3 + plane] cells, listed
  // at tile_list[pass][plane][tile * cap], cap kTileListY (luma) or
  // kTileListC (chroma).
  uint32_t *tile_count;
  uint32_t *tile_list[2][3];
  uint32_t tiles_x, tiles_y;
  int pw[3], ph[3];
};

// A segment into its grid cell and, for the tile kernel, into the list of
// every tile it runs in: a vertical-pass segment in the tiles whose columns
// its footprint reaches and whose rows widened by the halo hold its band, a
// horizontal-pass segment in the tile holding its band whose rows its
// footprint reaches (the host's index_tiles rule).  A picture the tile kernel
// takes has no two footprints overlapping and edges at least 8 samples apart,
// so a tile's list holds at most 24 bands x 12 luma (16 x 12 horizontal) or
// 24 x 6 chroma cells, within the caps.
struct GridEmit {
  const WalkParams *a;
  int d, p;
  __device__ void operator()(const EdgeSeg &s) const {
    const bool vert = s.flags & 1;
    const int unit = p ? 2 : 4, pu = p ? 8 : 4;
    const uint32_t band = (uint32_t)((vert ? s.y : s.x) / unit), pos = (uint32_t)((vert ? s.x : s.y) / pu);
    const uint32_t slots = a->slots[d][p];
    if (band >= a->bands[d][p] || pos >= slots) return;
    const uint32_t cell = band * slots + pos;
    a->grid[d][p][cell] = s;
    if (!a->tile_count) return;
    const int tp = p ? kDeblockTile / 2 : kDeblockTile, halo = p ? kDeblockHaloC : kDeblockHaloY;
    const int along = vert ? a->pw[p] : a->ph[p], q = vert ? s.x : s.y, bc = vert ? s.y : s.x;
    const int fs = max(q - reach_d(s.mfl >> 4), 0), fe = min(q + reach_d(s.mfl & 15), along);
    if (fs >= fe) return;  // touches no sample of the plane
    int x0, x1, y0, y1;    // tile columns and rows
    if (vert) {
      x0 = fs / tp;
      x1 = (fe - 1) / tp;
      y0 = bc - halo < 0 ? 0 : (bc - halo) / tp;
      y1 = (bc + unit + halo - 1) / tp;
    } else {
      x0 = x1 = bc / tp;
      y0 = fs / tp;
      y1 = (fe - 1) / tp;
    }
    x1 = min(x1, (int)a->tiles_x - 1);
    y1 = min(y1, (int)a->tiles_y - 1);
    const uint32_t cap = p ? kTileListC : kTileListY;
    for (int ty = y0; ty <= y1; ++ty)
      for (int tx = x0; tx <= x1; ++tx) {
        const uint32_t t = (uint32_t)ty * a->tiles_x + tx;
        const uint32_t k = atomicAdd(a->tile_count + t * 6 + d * 3 + p, 1u);
        if (k < cap) a->tile_list[d][p][(size_t)t * cap + k] = cell;
      }
  }
};

// Items of a list's first walk launch: its CU heads, then its tails, then
// (luma list) the motion records.
__host__ __device__ inline uint32_t unpack_items(const WalkParams &a, int list) {
  return a.n[list] + a.n_tails[list] + (list == 0 ? a.n_mv_recs : 0);
}

// Item i of list `list`: a CU head is copied into the CU's full record (the
// tail of a CU without TU map and TB split is never read, nor the motion of
// an intra CU) and the CU enters the CU map (CuGrid::build:
// cell -> CU covering it, the later CU winning, here the larger index); a
// tail or a motion record is copied into its CU's full record.  (The
// pictures the device walk takes have no overlapping CUs, so each cell is
// written by one CU: the crate's last-CU-wins rule needs no atomics.)
__device__ __forceinline__ void unpack_item(const WalkParams &a, int list, uint32_t i) {
  if (i < a.n[list]) {
    uint32_t cx, cy, cw, ch;
    if (a.compact[list]) {
      const uint4 v = reinterpret_cast<const uint4 *>(a.heads[list])[i];
      h266_deblock_cu &c = a.cus[list][i];
      cx = v.x & 0xFFFF;
      cy = v.x >> 16;
      cw = v.y & 0xFFFF;
      ch = v.y >> 16;
      c.x = cx;
      c.y = cy;
      c.w = cw;
      c.h = ch;
      c.qp_y = (int8_t)(v.z & 0xFF);
      const int q0 = (int8_t)((v.z >> 8) & 0xFF);
      c.qp_c[0] = q0 == -128 ? INT32_MIN : q0;
      c.qp_c[1] = (int8_t)((v.z >> 16) & 0xFF);
      c.qp_c[2] = (int8_t)(v.z >> 24);
      const uint32_t f = v.w & 0xFFFF;
      c.intra = f & 1;
      c.tu_y_coded = (f >> 1) & 1;
      c.tu_cb_coded = (f >> 2) & 1;
      c.tu_cr_coded = (f >> 3) & 1;
      c.bdpcm_luma = (f >> 4) & 1;
      c.bdpcm_chroma = (f >> 5) & 1;
      c.plt = (f >> 6) & 1;
      c.joint_cbcr2 = (f >> 7) & 1;
      c.ciip = (f >> 8) & 1;
      c.ibc = (f >> 9) & 1;
      c.has_num_sb = (f >> 10) & 1;
      c.has_tu64 = (f >> 11) & 1;
      c.has_tb_split = (f >> 12) & 1;
      c.num_sb_x = (v.w >> 16) & 0xFF;
      c.num_sb_y = v.w >> 24;
    } else {
      const uint64_t *src = reinterpret_cast<const uint64_t *>(a.heads[list] + (size_t)i * kCuHeadBytes);
      uint64_t *dst = reinterpret_cast<uint64_t *>(a.cus[list] + i);
      uint64_t w[kCuHeadBytes / 8];
#pragma unroll
      for (int k = 0; k < (int)(kCuHeadBytes / 8); ++k) w[k] = src[k];
#pragma unroll
      for (int k = 0; k < (int)(kCuHeadBytes / 8); ++k) dst[k] = w[k];
      cx = (uint32_t)w[0];
      cy = (uint32_t)(w[0] >> 32);
      cw = (uint32_t)w[1];
      ch = (uint32_t)(w[1] >> 32);
    }
    const int x0 = cx / 4, y0 = cy / 4;
    const int x1 = min((int)((cx + cw + 3) / 4), a.cw4), y1 = min((int)((cy + ch + 3) / 4), a.ch4);
    for (int y = y0; y < y1; ++y)
      for (int x = x0; x < x1; ++x) a.cu_grid[list][(size_t)y * a.cw4 + x] = (int32_t)i;  // CUs never overlap here
    return;
  }
  i -= a.n[list];
  if (i < a.n_tails[list]) {
    const CuTail &t = a.tails[list][i];
    if (t.index >= a.n[list]) return;
    const uint32_t *src = reinterpret_cast<const uint32_t *>(t.tail);
    uint32_t *dst = reinterpret_cast<uint32_t *>(reinterpret_cast<uint8_t *>(a.cus[list] + t.index) + kCuHeadBytes);
#pragma unroll
    for (int k = 0; k < 10; ++k) dst[k] = src[k];
    return;
  }
  i -= a.n_tails[list];
  if (list == 0 && i < a.n_mv_recs && a.mv_per_cu) {
    const CuMotionRec &r = a.mv_recs[i];
    if (r.index < a.n[0]) a.mv_per_cu[r.index] = r.m;
  }
}

__global__ void k_cu_grid(const __grid_constant__ WalkParams a, int list) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < unpack_items(a, list)) unpack_item(a, list, i);
}

// The edge walk of one CU for one (plane, pass) list (blockIdx.y = plane * 2 +
// pass) at one edge offset (blockIdx.z: offset / step; offsets beyond the CU
// return at once).
__global__ void __launch_bounds__(128) k_walk(const __grid_constant__ WalkParams a) {
  const int l = blockIdx.y, plane = l / 2, d = l % 2;
  const int list = plane ? 1 : 0;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n[list]) return;
  const h266_deblock_cu &cu = a.cus[list][i];
  const uint32_t step = plane ? 8 * (d == 0 ? a.cfg[plane].sub_w : a.cfg[plane].sub_h) : 4;
  const uint32_t off = blockIdx.z * step;
  if (off >= (d == 0 ? cu.w : cu.h)) return;
  const DevCuGrid grid{a.cu_grid[list], a.cw4, a.ch4};
  const GridEmit emit{&a, d, plane};
  if (plane == 0 && a.has_mv && a.mv_per_cu) {
    const CuMotion mv{&a.mv, a.mv_per_cu, DevCuGrid{a.cu_grid[0], a.cw4, a.ch4}};
    walk_cu(a.cus[list], grid, a.cfg[plane], d == 0, mv, a.nf[d], a.n_nf[d], i, emit, (int)off);
  } else {
    const MvGrid mv{plane == 0 && a.has_mv ? &a.mv : nullptr};
    walk_cu(a.cus[list], grid, a.cfg[plane], d == 0, mv, a.nf[d], a.n_nf[d], i, emit, (int)off);
  }
}

size_t align_up(size_t n) { return (n + 255) & ~(size_t)255; }

struct WalkLayout {
  size_t cu_grid[2], full[2], mv_full, grid[2][3], tile_count, tile_list[2][3], total;
  size_t zero_from, zero_end;  // [0, zero_from) is set to all ones (CU maps), [zero_from, zero_end) to zero
  uint32_t slots[2][3], bands[2][3];
};

WalkLayout walk_layout(const DeviceWalkIn &in) {
  // [CU maps: set to -1][tile counts: 0][segment grids: 0 when the strip
  // kernels scan them][full CU records, motion, tile lists: written before
  // they are read, not cleared]
  WalkLayout L{};
  const size_t cells = (size_t)((in.w + 3) / 4) * ((in.h + 3) / 4);
  size_t off = 0;
  for (int l = 0; l < 2; ++l) {
    L.cu_grid[l] = off;
    if (l == 0 || in.sep) off += align_up(cells * 4);
  }
  if (!in.sep) L.cu_grid[1] = L.cu_grid[0];
  L.zero_from = off;
  const size_t tiles = in.tile_lists ? (size_t)((in.w + kDeblockTile - 1) / kDeblockTile) *
                                           ((in.h + kDeblockTile - 1) / kDeblockTile)
                                     : 0;
  L.tile_count = off;
  off += align_up(tiles * 6 * sizeof(uint32_t));
  L.zero_end = off;
  for (int d = 0; d < 2; ++d)
    for (int p = 0; p < 3; ++p) {
      const bool has = p == 0 || in.cfi != 0;
      const int pw = p ? in.cw : in.w, ph = p ? in.ch : in.h;
      const int unit = p ? 2 : 4, pu = p ? 8 : 4;
      L.bands[d][p] = has && pw > 0 && ph > 0 ? (uint32_t)(((d == 0 ? ph : pw) + unit - 1) / unit) : 0;
      L.slots[d][p] = has && pw > 0 && ph > 0 ? (uint32_t)(((d == 0 ? pw : ph) + pu - 1) / pu) : 0;
      L.grid[d][p] = off;
      off += align_up((size_t)L.bands[d][p] * L.slots[d][p] * sizeof(EdgeSeg));
    }
  // The tile kernel reads only the cells the walk listed (and wrote); the
  // strip kernels scan every cell, so for them empty cells must read bS 0.
  if (!in.tiles_consume) L.zero_end = off;
  L.full[0] = off;
  off += align_up((size_t)in.n_cus * sizeof(h266_deblock_cu));
  L.full[1] = in.sep ? off : L.full[0];
  if (in.sep) off += align_up((size_t)in.n_chroma * sizeof(h266_deblock_cu));
  L.mv_full = off;
  if (in.mv_by_cu) off += align_up((size_t)in.n_cus * sizeof(h266_deblock_mv_cell));
  for (int d = 0; d < 2; ++d)
    for (int p = 0; p < 3; ++p) {
      L.tile_list[d][p] = off;
      off += align_up(tiles * (p ? kTileListC : kTileListY) * sizeof(uint32_t));
    }
  L.total = off;
  return L;
}

}  // namespace

size_t device_walk_bytes(const DeviceWalkIn &in) { return walk_layout(in).total; }

namespace {

// The walk's parameters of one picture (CU maps and segment grids in
// `scratch`, laid out by walk_layout) and the grids the tile kernel scans.
void fill_walk(const DeviceWalkIn &in, uint8_t *scratch, WalkParams &a, DeviceWalkOut &out, WalkLayout &L) {
  L = walk_layout(in);
  std::memset(&a, 0, sizeof a);
  const bool sep = in.sep;
  a.cus[0] = reinterpret_cast<h266_deblock_cu *>(scratch + L.full[0]);
  a.cus[1] = reinterpret_cast<h266_deblock_cu *>(scratch + L.full[1]);
  a.n[0] = (uint32_t)in.n_cus;
  a.n[1] = (uint32_t)(sep ? in.n_chroma : in.n_cus);
  for (int l = 0; l < 2; ++l) {
    a.heads[l] = in.heads[sep ? l : 0];
    a.compact[l] = in.compact[sep ? l : 0] ? 1 : 0;
    a.tails[l] = in.tails[sep ? l : 0];
    a.n_tails[l] = (uint32_t)in.n_tails[sep ? l : 0];
  }
  a.mv_recs = in.mv_recs;
  a.n_mv_recs = (uint32_t)in.n_mv_recs;
  a.cw4 = (in.w + 3) / 4;
  a.ch4 = (in.h + 3) / 4;
  a.cu_grid[0] = reinterpret_cast<int32_t *>(scratch + L.cu_grid[0]);
  a.cu_grid[1] = reinterpret_cast<int32_t *>(scratch + L.cu_grid[1]);
  a.has_mv = in.mv_cells != nullptr || in.mv_by_cu;
  a.mv_per_cu = in.mv_by_cu ? reinterpret_cast<h266_deblock_mv_cell *>(scratch + L.mv_full) : nullptr;
  a.mv.cells = in.mv_cells;
  a.mv.cells_w = in.mv_w;
  a.mv.cells_h = in.mv_h;
  a.nf[0] = in.nf_cols;
  a.nf[1] = in.nf_rows;
  a.n_nf[0] = (uint32_t)in.n_cols;
  a.n_nf[1] = (uint32_t)in.n_rows;
  const h266_deblock_params &pr = in.params;
  const int bd = (int)pr.bit_depth;
  const uint32_t ctb = 1u << pr.ctb_log2_size_y;
  a.cfg[0] = PlaneCfg{0, 1, 1, pr.luma_beta_offset_div2, pr.luma_tc_offset_div2, 0, bd, ctb};
  a.cfg[1] = PlaneCfg{1, 2, 2, pr.cb_beta_offset_div2, pr.cb_tc_offset_div2, pr.chroma_qp_offset_cb, bd, ctb};
  a.cfg[2] = PlaneCfg{2, 2, 2, pr.cr_beta_offset_div2, pr.cr_tc_offset_div2, pr.chroma_qp_offset_cr, bd, ctb};
  for (int d = 0; d < 2; ++d)
    for (int p = 0; p < 3; ++p) {
      a.grid[d][p] = reinterpret_cast<EdgeSeg *>(scratch + L.grid[d][p]);
      a.slots[d][p] = L.slots[d][p];
      a.bands[d][p] = L.bands[d][p];
      out.grid[d][p] = a.grid[d][p];
      out.slots[d][p] = L.slots[d][p];
      out.bands[d][p] = L.bands[d][p];
      a.tile_list[d][p] = in.tile_lists ? reinterpret_cast<uint32_t *>(scratch + L.tile_list[d][p]) : nullptr;
      out.tile_list[d][p] = a.tile_list[d][p];
    }
  out.tiles_x = (uint32_t)((in.w + kDeblockTile - 1) / kDeblockTile);
  out.tiles_y = (uint32_t)((in.h + kDeblockTile - 1) / kDeblockTile);
  a.tile_count = in.tile_lists ? reinterpret_cast<uint32_t *>(scratch + L.tile_count) : nullptr;
  out.tile_count = a.tile_count;
  a.tiles_x = out.tiles_x;
  a.tiles_y = out.tiles_y;
  a.pw[0] = in.w;
  a.ph[0] = in.h;
  a.pw[1] = a.pw[2] = in.cw;
  a.ph[1] = a.ph[2] = in.ch;
}

}  // namespace

int launch_device_walk(cudaStream_t st, const DeviceWalkIn &in, uint8_t *scratch, DeviceWalkOut &out,
                       uint64_t *launches) {
  WalkParams a;
  WalkLayout L;
  fill_walk(in, scratch, a, out, L);
  const bool sep = in.sep;
  // CU maps to -1 (no CU); full CU records, motion and segment grids to 0 (bS 0: no segment)
  H266_CUDA(cudaMemsetAsync(scratch, 0xFF, L.zero_from, st));
  H266_CUDA(cudaMemsetAsync(scratch + L.zero_from, 0, L.zero_end - L.zero_from, st));
  const int lists = in.cfi != 0 ? 6 : 2;
  for (int l = 0; l < (sep && in.cfi != 0 ? 2 : 1); ++l) {
    const uint32_t items = unpack_items(a, l);
    if (!items) continue;
    k_cu_grid<<<(items + 127) / 128, 128, 0, st>>>(a, l);
    H266_CUDA(cudaGetLastError());
    ++*launches;
  }
  const uint32_t nmax = std::max(a.n[0], a.n[1]);
  // offsets per CU: at most max dimension / 4 (luma; chroma has fewer)
  uint32_t max_dim = 4;
  max_dim = std::max(max_dim, in.max_cu_dim);
  if (nmax) {
    k_walk<<<dim3((nmax + 127) / 128, lists, (max_dim + 3) / 4), 128, 0, st>>>(a);
    H266_CUDA(cudaGetLastError());
    ++*launches;
  }
  return H266_OK;
}

// ---------------------------------------------------------------- batched device walk
//
// The walks of many pictures in three launches: the clearing of every
// picture's CU maps (-1) and segment grids (bS 0), the CU maps, and the edge
// walk.  Per picture a WalkBatchItem (parameters, clear extents, the walk's
// list count and offsets); CTAs find their picture by binary search over
// per-launch prefix tables of CTA counts.
struct WalkBatchItem {
  WalkParams p;
  uint4 *clear;            // the picture's walk scratch
  uint32_t ff_vec, zero_vec;  // 16-byte words set to all ones, then to zero
  uint32_t lists;          // (plane, pass) lists of the walk: 6, or 2 without chroma
  uint32_t cu_lists;       // CU maps built: 1, or 2 for a separate chroma tree
};

namespace {

__device__ __forceinline__ int batch_pick(const uint32_t *first, int n, uint32_t b) {
  int lo = 0, hi = n;  // first[lo] <= b < first[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (first[mid] <= b) lo = mid;
    else hi = mid;
  }
  return lo;
}

constexpr int kClearVecPerCta = 256 * 8;

__global__ void __launch_bounds__(256) k_walk_clear_batch(const WalkBatchItem *__restrict__ items,
                                                          const uint32_t *__restrict__ first, int n) {
  const int p = batch_pick(first, n, blockIdx.x);
  const WalkBatchItem &it = items[p];
  const uint32_t base = (blockIdx.x - first[p]) * kClearVecPerCta, total = it.ff_vec + it.zero_vec;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t i = base + k * 256 + threadIdx.x;
    if (i < total) it.clear[i] = i < it.ff_vec ? make_uint4(~0u, ~0u, ~0u, ~0u) : make_uint4(0, 0, 0, 0);
  }
}

__global__ void __launch_bounds__(128) k_cu_grid_batch(const WalkBatchItem *__restrict__ items,
                                                       const uint32_t *__restrict__ first, int n) {
  const int p = batch_pick(first, n, blockIdx.x);
  const WalkParams &a = items[p].p;
  const uint32_t lb = blockIdx.x - first[p], b0 = (unpack_items(a, 0) + 127) / 128;
  const int list = lb < b0 ? 0 : 1;
  const uint32_t i = (lb - (list ? b0 : 0)) * 128 + threadIdx.x;
  if (i < unpack_items(a, list)) unpack_item(a, list, i);
}

// blockIdx.y = plane * 2 + pass, blockIdx.z = edge offset / step, as k_walk.
__global__ void __launch_bounds__(128) k_walk_batch(const WalkBatchItem *__restrict__ items,
                                                    const uint32_t *__restrict__ first, int n) {
  __shared__ WalkParams s;
  const int p = batch_pick(first, n, blockIdx.x);
  if (blockIdx.y >= items[p].lists) return;  // uniform per CTA
  static_assert(sizeof(WalkParams) % 4 == 0, "word copy");
  const uint32_t *src = reinterpret_cast<const uint32_t *>(&items[p].p);
  uint32_t *dst = reinterpret_cast<uint32_t *>(&s);
  for (int i = threadIdx.x; i < (int)(sizeof(WalkParams) / 4); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  const WalkParams &a = s;
  const int l = blockIdx.y, plane = l / 2, d = l % 2;
  const int list = plane ? 1 : 0;
  const bool vert = d == 0;
  const DevCuGrid grid{a.cu_grid[list], a.cw4, a.ch4};
  const GridEmit emit{&a, d, plane};
  auto with_mv = [&](auto &&f) {
    if (plane == 0 && a.has_mv && a.mv_per_cu) f(CuMotion{&a.mv, a.mv_per_cu, DevCuGrid{a.cu_grid[0], a.cw4, a.ch4}});
    else f(MvGrid{plane == 0 && a.has_mv ? &a.mv : nullptr});
  };
  if (blockIdx.z == 0) {
    // The CUs' own edges (offset 0), packed: lane j of a warp counts the
    // segments of CU base + j's edge, and the warp walks all 32 CUs'
    // segments one per lane per round, so lanes stay busy whatever the CU
    // sizes (no memo across segments: the same values, recomputed).
    __shared__ uint32_t s_pre[4][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t base = (blockIdx.x - first[p]) * blockDim.x + warp * 32, i = base + lane;
    uint32_t nseg = 0;
    if (i < a.n[list]) {
      const CuWalkGeo g = cu_walk_geo(a.cus[list][i], a.cfg[plane], vert, a.nf[d], a.n_nf[d]);
      if (!g.off_grid && g.filter_edge) nseg = (g.n_other + g.seg - 1) / g.seg;
    }
    uint32_t incl = nseg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    s_pre[warp][lane] = incl - nseg;
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    __syncwarp();
    for (uint32_t t = lane; t < total; t += 32) {
      const int j = band_of(s_pre[warp], t);  // the lane whose CU holds segment t
      const size_t idx = base + j;
      const CuWalkGeo g = cu_walk_geo(a.cus[list][idx], a.cfg[plane], vert, a.nf[d], a.n_nf[d]);
      const uint32_t k = (t - s_pre[warp][j]) * g.seg;
      with_mv([&](const auto &mv) {
        WalkMemo memo;
        walk_segment(a.cus[list], grid, a.cfg[plane], vert, mv, idx, g, 0, g.filter_edge, !g.chroma && g.filter_edge,
                     k, emit, memo);
      });
    }
    return;
  }
  // edges inside a CU (blockIdx.z = offset / step): one thread per CU
  const uint32_t i = (blockIdx.x - first[p]) * blockDim.x + threadIdx.x;
  if (i >= a.n[list]) return;
  const h266_deblock_cu &cu = a.cus[list][i];
  const uint32_t step = plane ? 8 * (vert ? a.cfg[plane].sub_w : a.cfg[plane].sub_h) : 4;
  const uint32_t off = blockIdx.z * step;
  if (off >= (vert ? cu.w : cu.h)) return;
  with_mv([&](const auto &mv) { walk_cu(a.cus[list], grid, a.cfg[plane], vert, mv, a.nf[d], a.n_nf[d], i, emit, (int)off); });
}

}  // namespace

size_t walk_batch_item_size() { return sizeof(WalkBatchItem); }

void fill_walk_batch_item(void *out, const DeviceWalkIn &in, uint8_t *scratch, DeviceWalkOut &g, WalkBatchCounts &c) {
  WalkBatchItem it;
  std::memset(&it, 0, sizeof it);
  WalkLayout L;
  fill_walk(in, scratch, it.p, g, L);
  const bool sep = in.sep;
  it.clear = reinterpret_cast<uint4 *>(scratch);
  it.ff_vec = (uint32_t)(L.zero_from / 16);  // the CU maps come first (256-byte sections)
  it.zero_vec = (uint32_t)((L.zero_end - L.zero_from) / 16);
  it.lists = in.cfi != 0 ? 6 : 2;
  it.cu_lists = sep && in.cfi != 0 ? 2 : 1;
  c.clear_ctas = (it.ff_vec + it.zero_vec + kClearVecPerCta - 1) / kClearVecPerCta;
  c.grid_ctas = (unpack_items(it.p, 0) + 127) / 128 + (it.cu_lists == 2 ? (unpack_items(it.p, 1) + 127) / 128 : 0);
  c.walk_ctas = (std::max(it.p.n[0], it.p.n[1]) + 127) / 128;
  c.offsets = (std::max<uint32_t>(4, in.max_cu_dim) + 3) / 4;
  std::memcpy(out, &it, sizeof it);
}

int launch_walk_batch(cudaStream_t st, const void *d_items, const uint32_t *d_first_clear,
                      const uint32_t *d_first_grid, const uint32_t *d_first_walk, int n, const WalkBatchCounts &total,
                      uint64_t *launches) {
  if (n <= 0) return H266_OK;
  const WalkBatchItem *items = static_cast<const WalkBatchItem *>(d_items);
  if (total.clear_ctas) {
    k_walk_clear_batch<<<total.clear_ctas, 256, 0, st>>>(items, d_first_clear, n);
    H266_CUDA(cudaGetLastError());
    ++*launches;
  }
  if (total.grid_ctas) {
    k_cu_grid_batch<<<total.grid_ctas, 128, 0, st>>>(items, d_first_grid, n);
    H266_CUDA(cudaGetLastError());
    ++*launches;
  }
  if (total.walk_ctas) {
    k_walk_batch<<<dim3(total.walk_ctas, 6, total.offsets), 128, 0, st>>>(items, d_first_walk, n);
    H266_CUDA(cudaGetLastError());
    ++*launches;
  }
  return H266_OK;
}

uint32_t fill_deblock_tile_params_grid(void *out, const DPlane src[3], const DPlane dst[3], const uint16_t *lut,
                                       int bit_depth, const DeviceWalkOut &g) {
  TileParams a;
  std::memset(&a, 0, sizeof a);
  for (int i = 0; i < 3; ++i) {
    a.src[i] = src[i];
    a.dst[i] = dst[i];
    for (int d = 0; d < 2; ++d) {
      a.n_bands[d][i] = g.bands[d][i];
      a.grid[d][i] = g.grid[d][i];
      a.grid_slots[d][i] = g.slots[d][i];
      a.grid_list[d][i] = g.tile_list[d][i];
    }
  }
  a.grid_count = g.tile_count;
  a.grid_mode = 1;
  a.lut = lut;
  a.tiles_x = g.tiles_x;
  a.tiles_y = g.tiles_y;
  a.maxv = (1 << bit_depth) - 1;
  tile_tma_maps(a);
  std::memcpy(out, &a, sizeof a);
  return g.tiles_x * g.tiles_y;
}

int launch_deblock_tiles_grid(cudaStream_t st, const DPlane src[3], const DPlane dst[3], const uint16_t *lut,
                              int bit_depth, const DeviceWalkOut &g, uint64_t *launches) {
  TileParams a;
  std::memset(&a, 0, sizeof a);
  for (int i = 0; i < 3; ++i) {
    a.src[i] = src[i];
    a.dst[i] = dst[i];
    for (int d = 0; d < 2; ++d) {
      a.n_bands[d][i] = g.bands[d][i];
      a.grid[d][i] = g.grid[d][i];
      a.grid_slots[d][i] = g.slots[d][i];
      a.grid_list[d][i] = g.tile_list[d][i];
    }
  }
  a.grid_count = g.tile_count;
  a.grid_mode = 1;
  a.lut = lut;
  a.tiles_x = g.tiles_x;
  a.tiles_y = g.tiles_y;
  a.maxv = (1 << bit_depth) - 1;
  tile_tma_maps(a);
  const uint64_t n = (uint64_t)g.tiles_x * g.tiles_y;
  if (!n) return H266_OK;
  H266_TRY(prepare_tile_kernels());
  k_deblock_tiles<<<(unsigned)n, kTileThreads, kTileSmem, st>>>(a);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

}  // namespace h266
