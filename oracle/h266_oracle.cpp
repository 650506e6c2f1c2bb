// Oracle: a line-by-line CPU restatement of the oxideav-h266 (v0.0.8) in-loop
// filter chain, used ONLY as test infrastructure: the parity tests, the smoke
// check and bench.py's CPU-baseline leg call it as the checker.  Nothing in
// the product links or calls this file.
//
// Each function cites the reference function it restates (path:line within
// the crate).  The restatement keeps the reference's evaluation order (CU
// decode order, in-place sequential edge filtering, pre-SAO / pre-ALF
// snapshots) and its quirks, so its output is the reference's output on the
// same inputs.  Rust's `x << k` on possibly negative values is written `x * 2^k`
// (same result, no C++ undefined behaviour); `>>` on i32 is arithmetic in both.
//
// Environment switches of the reference (H266_DBG_*) are taken as unset.
#include "oxideav_h266_b200.h"
#include "spec_tables.h"

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace oracle {

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int64_t clampl(int64_t v, int64_t lo, int64_t hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int absi(int v) { return v < 0 ? -v : v; }

// ---------------------------------------------------------------------------
// deblock.rs
// ---------------------------------------------------------------------------

// TbSplit::tb_index, src/deblock.rs:297-305
static int tb_index(const h266_tb_split &ts, uint32_t rel) {
  int idx = 0;
  for (int i = 0; i < ts.n_bounds; ++i)
    if (rel >= ts.bounds[i]) idx = i + 1;
  return idx;
}
// TbSplit::tb_extent, src/deblock.rs:308-320
static void tb_extent(const h266_tb_split &ts, uint32_t rel, uint32_t dim, uint32_t &start, uint32_t &end) {
  start = 0;
  end = dim;
  for (int i = 0; i < ts.n_bounds; ++i) {
    uint32_t b = ts.bounds[i];
    if (rel < b) {
      end = b;
      break;
    }
    start = b;
  }
}

// DeblockCu::tu_coded_at, src/deblock.rs:168-200
static bool tu_coded_at(const h266_deblock_cu &cu, uint32_t c_idx, int lx, int ly) {
  if (cu.has_tu64) {
    uint32_t rx = (uint32_t)clampi(lx - (int)cu.x, 0, (int)cu.w - 1);
    uint32_t ry = (uint32_t)clampi(ly - (int)cu.y, 0, (int)cu.h - 1);
    uint32_t tx = std::min(rx / 64, 1u), ty = std::min(ry / 64, 1u);
    if (c_idx == 0) return cu.tu64.y[ty][tx];
    if (c_idx == 1) return cu.tu64.cb[ty][tx];
    return cu.tu64.cr[ty][tx];
  }
  if (cu.has_tb_split) {
    const h266_tb_split &ts = cu.tb_split;
    if (c_idx == 0 || !ts.luma_only) {
      uint32_t rel = ts.vertical ? (uint32_t)clampi(lx - (int)cu.x, 0, (int)cu.w - 1)
                                 : (uint32_t)clampi(ly - (int)cu.y, 0, (int)cu.h - 1);
      int idx = tb_index(ts, rel);
      if (c_idx == 0) return ts.y_coded[idx];
      if (c_idx == 1) return ts.cb_coded[idx];
      return ts.cr_coded[idx];
    }
  }
  if (c_idx == 0) return cu.tu_y_coded;
  if (c_idx == 1) return cu.tu_cb_coded;
  return cu.tu_cr_coded;
}

// DeblockCu::luma_tb_len, src/deblock.rs:206-223
static uint32_t luma_tb_len(const h266_deblock_cu &cu, int lx, int ly, bool vertical) {
  uint32_t dim = vertical ? cu.w : cu.h;
  uint32_t rel = vertical ? (uint32_t)clampi(lx - (int)cu.x, 0, (int)cu.w - 1)
                          : (uint32_t)clampi(ly - (int)cu.y, 0, (int)cu.h - 1);
  if (cu.has_tu64 && dim > 64) return std::min(dim - (rel / 64) * 64, 64u);
  if (cu.has_tb_split && (bool)cu.tb_split.vertical == vertical) {
    uint32_t s, e;
    tb_extent(cu.tb_split, rel, dim, s, e);
    return e - s;
  }
  return dim;
}

// DeblockCu::chroma_tb_len, src/deblock.rs:229-249
static uint32_t chroma_tb_len(const h266_deblock_cu &cu, int lx, int ly, bool vertical, uint32_t sub) {
  uint32_t dim = vertical ? cu.w : cu.h;
  uint32_t rel = vertical ? (uint32_t)clampi(lx - (int)cu.x, 0, (int)cu.w - 1)
                          : (uint32_t)clampi(ly - (int)cu.y, 0, (int)cu.h - 1);
  uint32_t luma_len;
  if (cu.has_tu64 && dim > 64) {
    luma_len = std::min(dim - (rel / 64) * 64, 64u);
  } else if (cu.has_tb_split) {
    if ((bool)cu.tb_split.vertical == vertical && !cu.tb_split.luma_only) {
      uint32_t s, e;
      tb_extent(cu.tb_split, rel, dim, s, e);
      luma_len = e - s;
    } else {
      luma_len = dim;
    }
  } else {
    luma_len = dim;
  }
  return luma_len / std::max(sub, 1u);
}

// DeblockCu::is_luma_tb_boundary, src/deblock.rs:253-270
static bool is_luma_tb_boundary(const h266_deblock_cu &cu, uint32_t off, bool vertical) {
  if (off == 0) return false;
  uint32_t dim = vertical ? cu.w : cu.h;
  if (off >= dim) return false;
  if (cu.has_tu64 && dim > 64) return off % 64 == 0;
  if (cu.has_tb_split && (bool)cu.tb_split.vertical == vertical) {
    for (int i = 0; i < cu.tb_split.n_bounds; ++i)
      if (cu.tb_split.bounds[i] == off) return true;
    return false;
  }
  return false;
}

// DeblockCu::is_chroma_tb_boundary, src/deblock.rs:274-291
static bool is_chroma_tb_boundary(const h266_deblock_cu &cu, uint32_t off, bool vertical) {
  if (off == 0) return false;
  uint32_t dim = vertical ? cu.w : cu.h;
  if (off >= dim) return false;
  if (cu.has_tu64 && dim > 64) return off % 64 == 0;
  if (cu.has_tb_split && (bool)cu.tb_split.vertical == vertical && !cu.tb_split.luma_only) {
    for (int i = 0; i < cu.tb_split.n_bounds; ++i)
      if (cu.tb_split.bounds[i] == off) return true;
    return false;
  }
  return false;
}

// DeblockMvGrid::at_luma, src/deblock.rs:353-363
static h266_deblock_mv_cell mv_at(const h266_deblock_mv_grid *g, int x, int y) {
  h266_deblock_mv_cell d;
  std::memset(&d, 0, sizeof d);
  if (x < 0 || y < 0) return d;
  uint64_t cx = (uint64_t)x / 4, cy = (uint64_t)y / 4;
  if (cx >= g->cells_w || cy >= g->cells_h) return d;
  return g->cells[cy * g->cells_w + cx];
}

// Table 43, src/deblock.rs:401-418
static const int kBetaPrime[64] = {0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,
                                   6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18, 20, 22, 24,
                                   26, 28, 30, 32, 34, 36, 38, 40, 42, 44, 46, 48, 50, 52, 54, 56,
                                   58, 60, 62, 64, 66, 68, 70, 72, 74, 76, 78, 80, 82, 84, 86, 88};
static const int kTcPrime[66] = {0,   0,   0,   0,   0,   0,   0,   0,   0,   0,   0,   0,   0,   0,
                                 0,   0,   0,   0,   3,   4,   4,   4,   4,   5,   5,   5,   5,   7,
                                 7,   8,   9,   10,  10,  11,  13,  14,  15,  17,  19,  21,  24,  25,
                                 29,  33,  36,  41,  45,  51,  57,  64,  71,  80,  89,  100, 112, 125,
                                 141, 157, 177, 198, 222, 250, 280, 314, 352, 395};

// beta_prime / tc_prime, src/deblock.rs:424-434
int beta_prime(int q) { return kBetaPrime[clampi(q, 0, 63)]; }
int tc_prime(int q) { return kTcPrime[clampi(q, 0, 65)]; }
// scale_tc_for_bit_depth, src/deblock.rs:439-446
int scale_tc(int tcp, uint32_t bd) {
  if (bd < 10) {
    int shift = 9 - (int)bd;
    return (tcp + (1 << shift)) >> (10 - (int)bd);
  }
  return tcp * (1 << ((int)bd - 10));
}
// scale_beta_for_bit_depth, src/deblock.rs:450-452
int scale_beta(int bp, uint32_t bd) { return bp * (1 << ((int)bd - 8)); }

struct Plane {
  uint16_t *s;
  size_t stride;
  int w, h;
  uint32_t bd;
};
static Plane mk(const h266_plane &p) { return Plane{p.samples, (size_t)p.stride, (int)p.width, (int)p.height, p.bit_depth}; }

// PlaneCtx, src/deblock.rs:458-474
struct PlaneCtx {
  Plane plane;
  uint32_t c_idx, sub_w, sub_h;
  int beta_offset_div2, tc_offset_div2, qp_offset;
  uint32_t bit_depth, ctb_size_y;
};

// CuGrid, src/deblock.rs:630-671
struct CuGrid {
  std::vector<int64_t> cells;  // -1 = None
  size_t cw = 0, ch = 0;
  void build(size_t pw, size_t ph, const h266_deblock_cu *cus, size_t n) {
    cw = (pw + 3) / 4;
    ch = (ph + 3) / 4;
    cells.assign(cw * ch, -1);
    for (size_t idx = 0; idx < n; ++idx) {
      const h266_deblock_cu &cu = cus[idx];
      size_t x0 = cu.x / 4, y0 = cu.y / 4;
      size_t x1 = std::min<size_t>(((size_t)cu.x + cu.w + 3) / 4, cw);
      size_t y1 = std::min<size_t>(((size_t)cu.y + cu.h + 3) / 4, ch);
      for (size_t cy = y0; cy < y1; ++cy)
        for (size_t cx = x0; cx < x1; ++cx) cells[cy * cw + cx] = (int64_t)idx;
    }
  }
  int64_t cu_at(int lx, int ly) const {
    if (lx < 0 || ly < 0) return -1;
    size_t cx = (size_t)lx / 4, cy = (size_t)ly / 4;
    if (cx >= cw || cy >= ch) return -1;
    return cells[cy * cw + cx];
  }
};

// bs_motion_rule, src/deblock.rs:992-1045
static bool bs_motion_rule(const h266_deblock_mv_cell &p, const h266_deblock_mv_cell &q) {
  uint32_t np = (p.pred_l0 ? 1u : 0u) + (p.pred_l1 ? 1u : 0u);
  uint32_t nq = (q.pred_l0 ? 1u : 0u) + (q.pred_l1 ? 1u : 0u);
  if (np != nq) return true;
  if (np == 0) return false;
  auto diff_ge8 = [](const int32_t *a, const int32_t *b) {
    return absi(a[0] - b[0]) >= 8 || absi(a[1] - b[1]) >= 8;
  };
  if (np == 1) {
    int p_poc = p.pred_l0 ? p.poc_l0 : p.poc_l1;
    const int32_t *p_mv = p.pred_l0 ? p.mv_l0 : p.mv_l1;
    int q_poc = q.pred_l0 ? q.poc_l0 : q.poc_l1;
    const int32_t *q_mv = q.pred_l0 ? q.mv_l0 : q.mv_l1;
    if (p_poc != q_poc) return true;
    return diff_ge8(p_mv, q_mv);
  }
  bool same_ordered = p.poc_l0 == q.poc_l0 && p.poc_l1 == q.poc_l1;
  bool same_swapped = p.poc_l0 == q.poc_l1 && p.poc_l1 == q.poc_l0;
  if (!(same_ordered || same_swapped)) return true;
  if (p.poc_l0 != p.poc_l1) {
    if (same_ordered && (diff_ge8(p.mv_l0, q.mv_l0) || diff_ge8(p.mv_l1, q.mv_l1))) return true;
    if (!same_ordered && (diff_ge8(p.mv_l0, q.mv_l1) || diff_ge8(p.mv_l1, q.mv_l0))) return true;
    return false;
  }
  bool straight = diff_ge8(p.mv_l0, q.mv_l0) || diff_ge8(p.mv_l1, q.mv_l1);
  bool crossed = diff_ge8(p.mv_l0, q.mv_l1) || diff_ge8(p.mv_l1, q.mv_l0);
  return straight && crossed;
}

// derive_bs, src/deblock.rs:1055-1119
static int derive_bs(uint32_t c_idx, const h266_deblock_cu &p, const h266_deblock_cu &q,
                     const h266_deblock_mv_grid *mv, int px, int py, int qx, int qy, bool is_tb_edge,
                     bool edge_idc2) {
  if (c_idx == 0 && p.bdpcm_luma && q.bdpcm_luma) return 0;
  if (c_idx != 0 && p.bdpcm_chroma && q.bdpcm_chroma) return 0;
  if (p.intra || q.intra) return 2;
  if (p.ciip || q.ciip) return 2;
  if (is_tb_edge) {
    if (tu_coded_at(p, c_idx, px, py) || tu_coded_at(q, c_idx, qx, qy)) return 1;
  }
  if (c_idx != 0 || !edge_idc2) return 0;
  if ((bool)p.ibc != (bool)q.ibc) return 1;
  if (p.ibc && q.ibc) {
    if (mv) {
      h266_deblock_mv_cell a = mv_at(mv, px, py), b = mv_at(mv, qx, qy);
      if (absi(a.mv_l0[0] - b.mv_l0[0]) >= 8 || absi(a.mv_l0[1] - b.mv_l0[1]) >= 8) return 1;
    }
    return 0;
  }
  if (mv) {
    if (bs_motion_rule(mv_at(mv, px, py), mv_at(mv, qx, qy))) return 1;
  }
  return 0;
}

// compute_thresholds_luma, src/deblock.rs:1122-1136
static void thresholds_luma(const PlaneCtx &pc, const h266_deblock_cu &p, const h266_deblock_cu &q, int bs,
                            int &beta, int &tc) {
  int qp = ((p.qp_y + q.qp_y + 1) >> 1) + 0;
  int q_beta = clampi(qp + pc.beta_offset_div2 * 2, 0, 63);
  beta = scale_beta(beta_prime(q_beta), pc.bit_depth);
  int q_tc = clampi(qp + 2 * (bs - 1) + pc.tc_offset_div2 * 2, 0, 65);
  tc = scale_tc(tc_prime(q_tc), pc.bit_depth);
}

// compute_thresholds_chroma, src/deblock.rs:1144-1174
static void thresholds_chroma(const PlaneCtx &pc, const h266_deblock_cu &p, const h266_deblock_cu &q, int bs,
                              int &beta, int &tc) {
  auto pick = [&](const h266_deblock_cu &c) -> int {
    if (c.qp_c[0] == INT32_MIN) return clampi(c.qp_y + pc.qp_offset, 0, 63);
    if (c.joint_cbcr2) return c.qp_c[2];
    uint32_t i = pc.c_idx >= 1 ? pc.c_idx - 1 : 0;
    return c.qp_c[std::min(i, 1u)];
  };
  int qp_c = (pick(p) + pick(q) + 1) >> 1;
  int q_beta = clampi(qp_c + pc.beta_offset_div2 * 2, 0, 63);
  beta = scale_beta(beta_prime(q_beta), pc.bit_depth);
  int q_tc = clampi(qp_c + 2 * (bs - 1) + pc.tc_offset_div2 * 2, 0, 65);
  tc = scale_tc(tc_prime(q_tc), pc.bit_depth);
}

// read_clamped / write, src/deblock.rs:1186-1200
static inline int rd(const Plane &pl, int x, int y) {
  int cx = clampi(x, 0, pl.w - 1), cy = clampi(y, 0, pl.h - 1);
  return pl.s[(size_t)cy * pl.stride + cx];
}
static inline void wr(Plane &pl, int x, int y, int v, uint32_t bd) {
  if (x < 0 || y < 0 || x >= pl.w || y >= pl.h) return;
  int mx = (1 << bd) - 1;
  pl.s[(size_t)y * pl.stride + x] = (uint16_t)clampi(v, 0, mx);
}

struct LumaDec {
  uint32_t d_e, d_ep, d_eq, mfl_p, mfl_q;
};

// luma_edge_decision, src/deblock.rs:1224-1409
static LumaDec luma_edge_decision(const Plane &pl, int cx, int cy, int beta, int tc, uint32_t mfl_p,
                                  uint32_t mfl_q, bool vert, bool ctb_row_edge) {
  auto P = [&](int i, int k) { return vert ? rd(pl, cx - i - 1, cy + k) : rd(pl, cx + k, cy - i - 1); };
  auto Q = [&](int j, int k) { return vert ? rd(pl, cx + j, cy + k) : rd(pl, cx + k, cy + j); };
  int dp0 = absi(P(2, 0) - 2 * P(1, 0) + P(0, 0));
  int dp3 = absi(P(2, 3) - 2 * P(1, 3) + P(0, 3));
  int dq0 = absi(Q(2, 0) - 2 * Q(1, 0) + Q(0, 0));
  int dq3 = absi(Q(2, 3) - 2 * Q(1, 3) + Q(0, 3));
  int sp0 = absi(P(3, 0) - P(0, 0));
  int sq0 = absi(Q(0, 0) - Q(3, 0));
  int spq0 = absi(P(0, 0) - Q(0, 0));
  int sp3 = absi(P(3, 3) - P(0, 3));
  int sq3 = absi(Q(0, 3) - Q(3, 3));
  int spq3 = absi(P(0, 3) - Q(0, 3));
  bool side_p_large = mfl_p > 3;
  bool side_q_large = mfl_q > 3;
  if (ctb_row_edge) side_p_large = false;
  bool d_sam0 = false, d_sam3 = false;
  if (side_p_large || side_q_large) {
    int dp0_l, dp3_l;
    if (side_p_large) {
      dp0_l = (dp0 + absi(P(5, 0) - 2 * P(4, 0) + P(3, 0)) + 1) >> 1;
      dp3_l = (dp3 + absi(P(5, 3) - 2 * P(4, 3) + P(3, 3)) + 1) >> 1;
    } else {
      mfl_p = 3;
      dp0_l = dp0;
      dp3_l = dp3;
    }
    int dq0_l, dq3_l;
    if (side_q_large) {
      dq0_l = (dq0 + absi(Q(5, 0) - 2 * Q(4, 0) + Q(3, 0)) + 1) >> 1;
      dq3_l = (dq3 + absi(Q(5, 3) - 2 * Q(4, 3) + Q(3, 3)) + 1) >> 1;
    } else {
      dq0_l = dq0;
      dq3_l = dq3;
    }
    int sp0_l = sp0, sp3_l = sp3;
    if (mfl_p == 7) {
      sp0_l = sp0 + absi(P(7, 0) - P(6, 0) - P(5, 0) + P(4, 0));
      sp3_l = sp3 + absi(P(7, 3) - P(6, 3) - P(5, 3) + P(4, 3));
    }
    int sq0_l = sq0, sq3_l = sq3;
    if (mfl_q == 7) {
      sq0_l = sq0 + absi(Q(4, 0) - Q(5, 0) - Q(6, 0) + Q(7, 0));
      sq3_l = sq3 + absi(Q(4, 3) - Q(5, 3) - Q(6, 3) + Q(7, 3));
    }
    int dl = (dp0_l + dq0_l) + (dp3_l + dq3_l);
    if (dl < beta) {
      auto row_decision = [&](int k, int dpq_l, int sp_l, int sq_l, int spq) {
        int sp_in = side_p_large ? (sp_l + absi(P(3, k) - P((int)mfl_p, k)) + 1) >> 1 : sp_l;
        int sq_in = side_q_large ? (sq_l + absi(Q(3, k) - Q((int)mfl_q, k)) + 1) >> 1 : sq_l;
        int s_thr1 = (3 * beta) >> 5;
        int s_thr2 = beta >> 4;
        return 2 * dpq_l < s_thr2 && sp_in + sq_in < s_thr1 && spq < ((5 * tc + 1) >> 1);
      };
      d_sam0 = row_decision(0, dp0_l + dq0_l, sp0_l, sq0_l, spq0);
      d_sam3 = row_decision(3, dp3_l + dq3_l, sp3_l, sq3_l, spq3);
    }
  }
  if (d_sam0 && d_sam3) return LumaDec{3, 1, 1, mfl_p, mfl_q};
  int dpq0 = dp0 + dq0, dpq3 = dp3 + dq3, dp = dp0 + dp3, dq = dq0 + dq3, d = dpq0 + dpq3;
  uint32_t d_e = 0, d_ep = 0, d_eq = 0;
  bool s_sam0 = false, s_sam3 = false;
  if (d < beta && mfl_p > 2 && mfl_q > 2) {
    int s_thr1 = beta >> 3, s_thr2 = beta >> 2;
    auto short_row = [&](int dpq, int sp, int sq, int spq) {
      return 2 * dpq < s_thr2 && sp + sq < s_thr1 && spq < ((5 * tc + 1) >> 1);
    };
    s_sam0 = short_row(dpq0, sp0, sq0, spq0);
    s_sam3 = short_row(dpq3, sp3, sq3, spq3);
  }
  if (d < beta) {
    d_e = 1;
    if (s_sam0 && s_sam3) {
      d_e = 2;
      mfl_p = 3;
      mfl_q = 3;
    }
    if (mfl_p > 1 && mfl_q > 1) {
      if (dp < ((beta + (beta >> 1)) >> 3)) d_ep = 1;
      if (dq < ((beta + (beta >> 1)) >> 3)) d_eq = 1;
    }
    if (d_e == 1) {
      mfl_p = 1 + d_ep;
      mfl_q = 1 + d_eq;
    }
  }
  return LumaDec{d_e, d_ep, d_eq, mfl_p, mfl_q};
}

// long_luma_apply, src/deblock.rs:1519-1673
static void long_luma_apply(Plane &pl, int cx, int cy, int tc, uint32_t mfl_p, uint32_t mfl_q, bool vert,
                            bool plt_p, bool plt_q) {
  uint32_t bd = pl.bd;
  int p[8] = {0}, q[8] = {0};
  for (uint32_t i = 0; i <= mfl_p && i < 8; ++i) p[i] = vert ? rd(pl, cx - (int)i - 1, cy) : rd(pl, cx, cy - (int)i - 1);
  for (uint32_t j = 0; j <= mfl_q && j < 8; ++j) q[j] = vert ? rd(pl, cx + (int)j, cy) : rd(pl, cx, cy + (int)j);
  int ref_middle;
  if (mfl_p == 5 && mfl_q == 5) {
    ref_middle = (p[4] + p[3] + 2 * (p[2] + p[1] + p[0] + q[0] + q[1] + q[2]) + q[3] + q[4] + 8) >> 4;
  } else if (mfl_p == mfl_q) {
    ref_middle = (p[6] + p[5] + p[4] + p[3] + p[2] + p[1] + 2 * (p[0] + q[0]) + q[1] + q[2] + q[3] + q[4] + q[5] +
                  q[6] + 8) >> 4;
  } else if ((mfl_p == 7 && mfl_q == 5) || (mfl_p == 5 && mfl_q == 7)) {
    ref_middle = (p[5] + p[4] + p[3] + p[2] + 2 * (p[1] + p[0] + q[0] + q[1]) + q[2] + q[3] + q[4] + q[5] + 8) >> 4;
  } else if ((mfl_p == 5 && mfl_q == 3) || (mfl_p == 3 && mfl_q == 5)) {
    ref_middle = (p[3] + p[2] + p[1] + p[0] + q[0] + q[1] + q[2] + q[3] + 4) >> 3;
  } else if (mfl_p == 3 && mfl_q == 7) {
    ref_middle = (2 * (p[2] + p[1] + p[0] + q[0]) + p[0] + p[1] + q[1] + q[2] + q[3] + q[4] + q[5] + q[6] + 8) >> 4;
  } else {
    ref_middle = (p[6] + p[5] + p[4] + p[3] + p[2] + p[1] + 2 * (q[2] + q[1] + q[0] + p[0]) + q[0] + q[1] + 8) >> 4;
  }
  int ref_p = (p[mfl_p] + p[mfl_p - 1] + 1) >> 1;
  int ref_q = (q[mfl_q] + q[mfl_q - 1] + 1) >> 1;
  static const int F7[7] = {59, 50, 41, 32, 23, 14, 5}, F5[5] = {58, 45, 32, 19, 6}, F3[3] = {53, 32, 11};
  static const int T7[7] = {6, 5, 4, 3, 2, 1, 1}, T5[5] = {6, 5, 4, 3, 2}, T3[3] = {6, 4, 2};
  const int *fi = mfl_p == 7 ? F7 : (mfl_p == 5 ? F5 : F3);
  const int *tp = mfl_p == 7 ? T7 : (mfl_p == 5 ? T5 : T3);
  const int *gj = mfl_q == 7 ? F7 : (mfl_q == 5 ? F5 : F3);
  const int *tq = mfl_q == 7 ? T7 : (mfl_q == 5 ? T5 : T3);
  for (uint32_t i = 0; i < mfl_p; ++i) {
    if (plt_p) break;
    int lo = p[i] - ((tc * tp[i]) >> 1), hi = p[i] + ((tc * tp[i]) >> 1);
    int v = clampi((ref_middle * fi[i] + ref_p * (64 - fi[i]) + 32) >> 6, lo, hi);
    if (vert) wr(pl, cx - (int)i - 1, cy, v, bd);
    else wr(pl, cx, cy - (int)i - 1, v, bd);
  }
  for (uint32_t j = 0; j < mfl_q; ++j) {
    if (plt_q) break;
    int lo = q[j] - ((tc * tq[j]) >> 1), hi = q[j] + ((tc * tq[j]) >> 1);
    int v = clampi((ref_middle * gj[j] + ref_q * (64 - gj[j]) + 32) >> 6, lo, hi);
    if (vert) wr(pl, cx + (int)j, cy, v, bd);
    else wr(pl, cx, cy + (int)j, v, bd);
  }
}

// short_luma_apply, src/deblock.rs:1680-1776
static void short_luma_apply(Plane &pl, int cx, int cy, int tc, uint32_t d_e, uint32_t d_ep, uint32_t d_eq,
                             bool vert, bool plt_p, bool plt_q) {
  uint32_t bd = pl.bd;
  auto P = [&](int i) { return vert ? rd(pl, cx - i - 1, cy) : rd(pl, cx, cy - i - 1); };
  auto Q = [&](int j) { return vert ? rd(pl, cx + j, cy) : rd(pl, cx, cy + j); };
  int p3 = P(3), p2 = P(2), p1 = P(1), p0 = P(0), q0 = Q(0), q1 = Q(1), q2 = Q(2), q3 = Q(3);
  auto WP = [&](int i, int v) {
    if (vert) wr(pl, cx - i - 1, cy, v, bd);
    else wr(pl, cx, cy - i - 1, v, bd);
  };
  auto WQ = [&](int j, int v) {
    if (vert) wr(pl, cx + j, cy, v, bd);
    else wr(pl, cx, cy + j, v, bd);
  };
  if (d_e == 2) {
    int p0n = clampi((p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3, p0 - 3 * tc, p0 + 3 * tc);
    int p1n = clampi((p2 + p1 + p0 + q0 + 2) >> 2, p1 - 2 * tc, p1 + 2 * tc);
    int p2n = clampi((2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3, p2 - tc, p2 + tc);
    int q0n = clampi((p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3, q0 - 3 * tc, q0 + 3 * tc);
    int q1n = clampi((p0 + q0 + q1 + q2 + 2) >> 2, q1 - 2 * tc, q1 + 2 * tc);
    int q2n = clampi((p0 + q0 + q1 + 3 * q2 + 2 * q3 + 4) >> 3, q2 - tc, q2 + tc);
    if (!plt_p) {
      WP(0, p0n);
      WP(1, p1n);
      WP(2, p2n);
    }
    if (!plt_q) {
      WQ(0, q0n);
      WQ(1, q1n);
      WQ(2, q2n);
    }
  } else {
    int delta_raw = (9 * (q0 - p0) - 3 * (q1 - p1) + 8) >> 4;
    if (absi(delta_raw) < tc * 10) {
      int delta = clampi(delta_raw, -tc, tc);
      if (!plt_p) WP(0, p0 + delta);
      if (!plt_q) WQ(0, q0 - delta);
      if (d_ep == 1 && !plt_p) {
        int dp = clampi((((p2 + p0 + 1) >> 1) - p1 + delta) >> 1, -(tc >> 1), tc >> 1);
        WP(1, p1 + dp);
      }
      if (d_eq == 1 && !plt_q) {
        int dq = clampi((((q2 + q0 + 1) >> 1) - q1 - delta) >> 1, -(tc >> 1), tc >> 1);
        WQ(1, q1 + dq);
      }
    }
  }
}

// run_luma_filter, src/deblock.rs:1416-1508
static void run_luma_filter(Plane &pl, int cx, int cy, int beta, int tc, uint32_t mfl_p, uint32_t mfl_q, bool vert,
                            bool ctb_row_edge, bool plt_p, bool plt_q) {
  if (tc == 0) return;
  LumaDec dec = luma_edge_decision(pl, cx, cy, beta, tc, mfl_p, mfl_q, vert, ctb_row_edge);
  if (dec.d_e == 0) return;
  for (int k = 0; k < 4; ++k) {
    int x = vert ? cx : cx + k, y = vert ? cy + k : cy;
    if (dec.d_e == 3) long_luma_apply(pl, x, y, tc, dec.mfl_p, dec.mfl_q, vert, plt_p, plt_q);
    else short_luma_apply(pl, x, y, tc, dec.d_e, dec.d_ep, dec.d_eq, vert, plt_p, plt_q);
  }
}

// chroma_strong_decision_v / _h, src/deblock.rs:1932-1982 (the vertical form
// is the horizontal one along the other axis with short_p = false).
static bool chroma_strong_decision(const Plane &pl, int cx, int cy, int beta, int tc, bool vert, bool short_p) {
  auto A = [&](int d) { return vert ? rd(pl, cx + d, cy) : rd(pl, cx, cy + d); };
  int p1 = A(-2);
  int p3 = short_p ? p1 : A(-4);
  int p2 = short_p ? p1 : A(-3);
  int p0 = A(-1), q0 = A(0), q1 = A(1), q2 = A(2), q3 = A(3);
  int dp = absi(p2 - 2 * p1 + p0), dq = absi(q2 - 2 * q1 + q0);
  int dpq = 2 * (dp + dq);
  int edge = absi(p3 - p0) + absi(q0 - q3);
  int centre = absi(p0 - q0);
  return dpq < (beta >> 2) && edge < (beta >> 3) && centre < ((5 * tc + 1) >> 1);
}

// chroma_strong_apply_v / _h, src/deblock.rs:1986-2074
static void chroma_strong_apply(Plane &pl, int cx, int cy, int tc, uint32_t bd, bool vert, bool short_p, bool plt_p,
                                bool plt_q) {
  auto A = [&](int d) { return vert ? rd(pl, cx + d, cy) : rd(pl, cx, cy + d); };
  auto W = [&](int d, int v) {
    if (vert) wr(pl, cx + d, cy, v, bd);
    else wr(pl, cx, cy + d, v, bd);
  };
  int p1 = A(-2), p0 = A(-1), q0 = A(0), q1 = A(1), q2 = A(2), q3 = A(3);
  if (short_p) {
    int p0n = clampi((3 * p1 + 2 * p0 + q0 + q1 + q2 + 4) >> 3, p0 - tc, p0 + tc);
    int q0n = clampi((2 * p1 + p0 + 2 * q0 + q1 + q2 + q3 + 4) >> 3, q0 - tc, q0 + tc);
    int q1n = clampi((p1 + p0 + q0 + 2 * q1 + q2 + 2 * q3 + 4) >> 3, q1 - tc, q1 + tc);
    int q2n = clampi((p0 + q0 + q1 + 2 * q2 + 3 * q3 + 4) >> 3, q2 - tc, q2 + tc);
    if (!plt_p) W(-1, p0n);
    if (!plt_q) {
      W(0, q0n);
      W(1, q1n);
      W(2, q2n);
    }
    return;
  }
  int p3 = A(-4), p2 = A(-3);
  int p0n = clampi((p3 + p2 + p1 + 2 * p0 + q0 + q1 + q2 + 4) >> 3, p0 - tc, p0 + tc);
  int p1n = clampi((2 * p3 + p2 + 2 * p1 + p0 + q0 + q1 + 4) >> 3, p1 - tc, p1 + tc);
  int p2n = clampi((3 * p3 + 2 * p2 + p1 + p0 + q0 + 4) >> 3, p2 - tc, p2 + tc);
  int q0n = clampi((p2 + p1 + p0 + 2 * q0 + q1 + q2 + q3 + 4) >> 3, q0 - tc, q0 + tc);
  int q1n = clampi((p1 + p0 + q0 + 2 * q1 + q2 + 2 * q3 + 4) >> 3, q1 - tc, q1 + tc);
  int q2n = clampi((p0 + q0 + q1 + 2 * q2 + 3 * q3 + 4) >> 3, q2 - tc, q2 + tc);
  if (!plt_p) {
    W(-1, p0n);
    W(-2, p1n);
    W(-3, p2n);
  }
  if (!plt_q) {
    W(0, q0n);
    W(1, q1n);
    W(2, q2n);
  }
}

// run_chroma_filter_v / _h, src/deblock.rs:1803-1926
static void run_chroma_filter(Plane &pl, int cx, int cy, int beta, int tc, int bs, uint32_t mfl_p, uint32_t mfl_q,
                              bool vert, bool plt_p, bool plt_q) {
  if (tc == 0) return;
  if (mfl_p == 1 && mfl_q == 1 && bs != 2) return;
  uint32_t bd = pl.bd;
  bool strong_eligible, short_p;
  if (vert) {
    strong_eligible = mfl_p == 3 && mfl_q == 3;
    short_p = false;
  } else {
    strong_eligible = mfl_q == 3 && (mfl_p == 3 || mfl_p == 1);
    short_p = mfl_p == 1;
  }
  if (strong_eligible) {
    bool dec0 = chroma_strong_decision(pl, cx, cy, beta, tc, vert, short_p);
    bool dec1 = vert ? chroma_strong_decision(pl, cx, cy + 1, beta, tc, vert, short_p)
                     : chroma_strong_decision(pl, cx + 1, cy, beta, tc, vert, short_p);
    if (dec0 && dec1) {
      for (int k = 0; k <= 1; ++k) {
        if (vert) chroma_strong_apply(pl, cx, cy + k, tc, bd, vert, short_p, plt_p, plt_q);
        else chroma_strong_apply(pl, cx + k, cy, tc, bd, vert, short_p, plt_p, plt_q);
      }
      return;
    }
  }
  for (int k = 0; k < 2; ++k) {
    int x = vert ? cx : cx + k, y = vert ? cy + k : cy;
    auto A = [&](int d) { return vert ? rd(pl, x + d, y) : rd(pl, x, y + d); };
    int p1 = A(-2), p0 = A(-1), q0 = A(0), q1 = A(1);
    int delta = clampi(((q0 - p0) * 4 + p1 - q1 + 4) >> 3, -tc, tc);
    if (!plt_p) {
      if (vert) wr(pl, x - 1, y, p0 + delta, bd);
      else wr(pl, x, y - 1, p0 + delta, bd);
    }
    if (!plt_q) wr(pl, x, y, q0 - delta, bd);
  }
}

// One filtered edge segment in the reference's processing order; recorded
// for the edge-list tests (the filter itself is applied in place).
struct EdgeRec {
  int32_t c_idx, vertical, qx, qy;  // segment anchor: q0 in component samples
  int32_t bs, mfl_p, mfl_q, beta, tc, ctb_row, plt_p, plt_q;
  int32_t cu_idx, off;
};

// deblock_cu_dir, src/deblock.rs:707-983
static void deblock_cu_dir(PlaneCtx &pc, const h266_deblock_cu *cus, const CuGrid &grid,
                           const h266_deblock_mv_grid *mv, uint32_t idx, const h266_deblock_cu &cu, bool vertical,
                           const uint32_t *no_filter, size_t n_no_filter, std::vector<EdgeRec> *log, bool apply) {
  uint32_t c_idx = pc.c_idx;
  if (c_idx != 0) {
    uint32_t lead_c = vertical ? cu.x / pc.sub_w : cu.y / pc.sub_h;
    if (lead_c % 8 != 0) return;
  }
  uint32_t n_cb = vertical ? cu.w : cu.h;
  uint32_t n_other = vertical ? cu.h : cu.w;
  uint32_t lead_luma = vertical ? cu.x : cu.y;
  bool excluded = false;
  for (size_t i = 0; i < n_no_filter; ++i)
    if (no_filter[i] == lead_luma) excluded = true;
  bool filter_edge = lead_luma != 0 && !excluded;
  uint32_t grid_step = c_idx == 0 ? 4u : 8u * (vertical ? pc.sub_w : pc.sub_h);
  uint32_t seg_step = c_idx == 0 ? 4u : 2u * (vertical ? pc.sub_h : pc.sub_w);
  uint32_t num_sb_axis = 1;
  if (c_idx == 0) {
    num_sb_axis = cu.has_num_sb ? (vertical ? cu.num_sb_x : cu.num_sb_y) : 1u;
    num_sb_axis = std::max(num_sb_axis, 1u);
  }
  uint32_t sb = std::max(8u, n_cb / num_sb_axis);
  uint32_t n8 = n_cb / 8;
  uint32_t last_sb_edge = std::min(std::max(n8, 1u) - 1, num_sb_axis - 1);
  uint32_t ctb_h_c = pc.ctb_size_y / std::max(pc.sub_h, 1u);

  for (uint32_t off = 0; off < n_cb; off += grid_step) {
    bool is_tb = off == 0 ? filter_edge
                          : (c_idx == 0 ? is_luma_tb_boundary(cu, off, vertical) : is_chroma_tb_boundary(cu, off, vertical));
    bool is_sb_edge = c_idx == 0 && off % sb == 0 && off / sb <= last_sb_edge && (off > 0 || filter_edge);
    if (!(is_tb || is_sb_edge)) continue;
    for (uint32_t k = 0; k < n_other; k += seg_step) {
      int qx = vertical ? (int)(cu.x + off) : (int)(cu.x + k);
      int qy = vertical ? (int)(cu.y + k) : (int)(cu.y + off);
      int px = vertical ? qx - 1 : qx, py = vertical ? qy : qy - 1;
      int64_t p_idx = off == 0 ? grid.cu_at(px, py) : (int64_t)idx;
      if (p_idx < 0) continue;
      if (off == 0 && p_idx == (int64_t)idx) continue;
      const h266_deblock_cu &p_cu = cus[p_idx];
      const h266_deblock_cu &q_cu = cu;
      int bs = derive_bs(c_idx, p_cu, q_cu, mv, px, py, qx, qy, is_tb, is_sb_edge);
      if (bs == 0) continue;
      if (c_idx == 0) {
        uint32_t mfl_p = 0, mfl_q = 0;
        if (is_tb) {
          uint32_t wq = luma_tb_len(q_cu, qx, qy, vertical);
          uint32_t wp = luma_tb_len(p_cu, px, py, vertical);
          if (wp <= 4 || wq <= 4) {
            mfl_p = 1;
            mfl_q = 1;
          } else {
            mfl_p = wp >= 32 ? 7 : 3;
            mfl_q = wq >= 32 ? 7 : 3;
          }
        }
        if (is_sb_edge) {
          if (off == 0) {
            if (num_sb_axis > 1) mfl_q = std::min(mfl_q, 5u);
            if (p_cu.has_num_sb) mfl_p = std::min(mfl_p, 5u);
          } else {
            auto tb_at = [&](int64_t z) -> bool {
              if (z < 0 || (uint64_t)z >= n_cb) return false;
              if (z == 0) return filter_edge;
              return is_luma_tb_boundary(cu, (uint32_t)z, vertical);
            };
            if (is_tb) {
              mfl_p = std::min(mfl_p, 5u);
              mfl_q = std::min(mfl_q, 5u);
            } else if (tb_at((int64_t)off - 4) || tb_at((int64_t)off + 4)) {
              mfl_p = 1;
              mfl_q = 1;
            } else if (off / sb == 1 || off / sb == std::max(n8, 1u) - 1 || tb_at((int64_t)off - sb) ||
                       tb_at((int64_t)off + sb)) {
              mfl_p = 2;
              mfl_q = 2;
            } else {
              mfl_p = 3;
              mfl_q = 3;
            }
          }
        }
        bool ctb_row_edge = !vertical && off == 0 && pc.ctb_size_y > 0 && cu.y % pc.ctb_size_y == 0;
        int beta, tc;
        thresholds_luma(pc, p_cu, q_cu, bs, beta, tc);
        if (log) log->push_back(EdgeRec{0, vertical, qx, qy, bs, (int)mfl_p, (int)mfl_q, beta, tc, ctb_row_edge,
                                        p_cu.plt, q_cu.plt, (int)idx, (int)off});
        if (apply) run_luma_filter(pc.plane, qx, qy, beta, tc, mfl_p, mfl_q, vertical, ctb_row_edge, p_cu.plt, q_cu.plt);
      } else {
        uint32_t sub_axis = vertical ? pc.sub_w : pc.sub_h;
        uint32_t wq = chroma_tb_len(q_cu, qx, qy, vertical, sub_axis);
        uint32_t wp = chroma_tb_len(p_cu, px, py, vertical, sub_axis);
        uint32_t mfl_p, mfl_q;
        if (wp >= 8 && wq >= 8) {
          bool ctb_row = !vertical && off == 0 && ctb_h_c > 0 && (cu.y / pc.sub_h) % ctb_h_c == 0;
          mfl_p = ctb_row ? 1 : 3;
          mfl_q = 3;
        } else {
          mfl_p = 1;
          mfl_q = 1;
        }
        int beta, tc;
        thresholds_chroma(pc, p_cu, q_cu, bs, beta, tc);
        int ex = qx / (int)pc.sub_w, ey = qy / (int)pc.sub_h;
        if (log) log->push_back(EdgeRec{(int)c_idx, vertical, ex, ey, bs, (int)mfl_p, (int)mfl_q, beta, tc, 0,
                                        p_cu.plt, q_cu.plt, (int)idx, (int)off});
        if (apply) run_chroma_filter(pc.plane, ex, ey, beta, tc, bs, mfl_p, mfl_q, vertical, p_cu.plt, q_cu.plt);
      }
    }
  }
}

// apply_deblocking_clipped, src/deblock.rs:497-617
static void apply_deblocking_clipped(h266_picture *out, const h266_deblock_cu *cus, size_t n_cus,
                                     const h266_deblock_cu *chroma_cus, size_t n_chroma, const h266_deblock_mv_grid *mv,
                                     const h266_deblock_params *params, uint32_t cfi, const uint32_t *nf_cols,
                                     size_t n_cols, const uint32_t *nf_rows, size_t n_rows,
                                     std::vector<EdgeRec> *log, bool apply) {
  if (params->disabled) return;
  CuGrid grid;
  grid.build(out->luma.width, out->luma.height, cus, n_cus);
  CuGrid cgrid;
  if (chroma_cus) cgrid.build(out->luma.width, out->luma.height, chroma_cus, n_chroma);
  uint32_t ctb = 1u << params->ctb_log2_size_y;
  PlaneCtx luma{mk(out->luma), 0, 1, 1, params->luma_beta_offset_div2, params->luma_tc_offset_div2, 0,
                params->bit_depth, ctb};
  for (int dir = 0; dir < 2; ++dir) {
    bool vertical = dir == 0;
    for (size_t i = 0; i < n_cus; ++i)
      deblock_cu_dir(luma, cus, grid, mv, (uint32_t)i, cus[i], vertical, vertical ? nf_cols : nf_rows,
                     vertical ? n_cols : n_rows, log, apply);
  }
  if (cfi != 0) {
    const h266_deblock_cu *c_cus = chroma_cus ? chroma_cus : cus;
    size_t n_c = chroma_cus ? n_chroma : n_cus;
    const CuGrid &cg = chroma_cus ? cgrid : grid;
    PlaneCtx cb{mk(out->cb), 1, 2, 2, params->cb_beta_offset_div2, params->cb_tc_offset_div2,
                params->chroma_qp_offset_cb, params->bit_depth, ctb};
    PlaneCtx cr{mk(out->cr), 2, 2, 2, params->cr_beta_offset_div2, params->cr_tc_offset_div2,
                params->chroma_qp_offset_cr, params->bit_depth, ctb};
    PlaneCtx *pcs[2] = {&cb, &cr};
    for (PlaneCtx *pc : pcs)
      for (int dir = 0; dir < 2; ++dir) {
        bool vertical = dir == 0;
        for (size_t i = 0; i < n_c; ++i)
          deblock_cu_dir(*pc, c_cus, cg, nullptr, (uint32_t)i, c_cus[i], vertical, vertical ? nf_cols : nf_rows,
                         vertical ? n_cols : n_rows, log, apply);
      }
  }
}

// ---------------------------------------------------------------------------
// sao.rs
// ---------------------------------------------------------------------------

// SaoConfig::chroma_subsampling src/sao.rs:344-351 and AlfConfig::chroma_subsampling src/alf.rs:161-168
static void chroma_sub(uint32_t cfi, int &sw, int &sh) {
  if (cfi == 1) { sw = 2; sh = 2; }
  else if (cfi == 2) { sw = 2; sh = 1; }
  else { sw = 1; sh = 1; }
}

// `span` closure of apply_sao_clipped src/sao.rs:429-436 / clip_rect_for_ctb src/alf.rs:1084-1091
static void span(const uint32_t *bds, size_t n, uint32_t v, int mx, int &lo, int &hi) {
  for (size_t i = 0; i + 1 < n; ++i) {
    if (v >= bds[i] && v < bds[i + 1]) {
      lo = (int)bds[i];
      hi = std::min((int)bds[i + 1], mx);
      return;
    }
  }
  lo = 0;
  hi = mx;
}

static inline int sgn(int x) { return x < 0 ? -1 : (x > 0 ? 1 : 0); }

// apply_sao_ctb, src/sao.rs:504-626
static void apply_sao_ctb(Plane &pl, const uint16_t *pre, bool has_clip, const int clip[4], uint32_t rx, uint32_t ry,
                          uint32_t nw, uint32_t nh, uint32_t bd, const h266_sao_ctb &prm) {
  size_t x_ctb = (size_t)rx * nw, y_ctb = (size_t)ry * nh;
  size_t stride = pl.stride;
  int pw = pl.w, ph = pl.h;
  size_t i_max = std::min<size_t>(nw, (size_t)pl.w > x_ctb ? pl.w - x_ctb : 0);
  size_t j_max = std::min<size_t>(nh, (size_t)pl.h > y_ctb ? pl.h - y_ctb : 0);
  int max_val = (1 << bd) - 1;
  if (prm.sao_type_idx == 2) {
    static const int H0[4] = {-1, 0, -1, 1}, V0[4] = {0, -1, -1, -1}, H1[4] = {1, 0, 1, -1}, V1[4] = {0, 1, 1, 1};
    int c = prm.eo_class & 3;
    for (size_t j = 0; j < j_max; ++j)
      for (size_t i = 0; i < i_max; ++i) {
        int xs = (int)(x_ctb + i), ys = (int)(y_ctb + j);
        int nx0 = xs + H0[c], ny0 = ys + V0[c], nx1 = xs + H1[c], ny1 = ys + V1[c];
        bool outside = nx0 < 0 || ny0 < 0 || nx1 < 0 || ny1 < 0 || nx0 >= pw || ny0 >= ph || nx1 >= pw || ny1 >= ph;
        if (has_clip)
          outside = outside || nx0 < clip[0] || ny0 < clip[1] || nx1 < clip[0] || ny1 < clip[1] || nx0 >= clip[2] ||
                    ny0 >= clip[3] || nx1 >= clip[2] || ny1 >= clip[3];
        size_t at = (size_t)ys * stride + xs;
        if (outside) {
          pl.s[at] = (uint16_t)clampi(pre[at], 0, max_val);
          continue;
        }
        int p = pre[at];
        int n0 = pre[(size_t)ny0 * stride + nx0], n1 = pre[(size_t)ny1 * stride + nx1];
        int e = 2 + sgn(p - n0) + sgn(p - n1);
        if (e <= 2) e = e == 2 ? 0 : e + 1;
        int off = (e >= 1 && e <= 4) ? prm.offset_val[e] : 0;
        pl.s[at] = (uint16_t)clampi(p + off, 0, max_val);
      }
  } else if (prm.sao_type_idx == 1) {
    int band_shift = (int)bd - 5;
    int band_table[32] = {0};
    int left = prm.band_position;
    for (int k = 0; k < 4; ++k) band_table[(k + left) & 31] = k + 1;
    for (size_t j = 0; j < j_max; ++j)
      for (size_t i = 0; i < i_max; ++i) {
        size_t at = (y_ctb + j) * stride + x_ctb + i;
        int p = pre[at];
        int bi = band_shift >= 0 ? band_table[(p >> band_shift) & 31] : band_table[p & 31];
        int off = (bi >= 1 && bi <= 4) ? prm.offset_val[bi] : 0;
        pl.s[at] = (uint16_t)clampi(p + off, 0, max_val);
      }
  }
}

static std::vector<uint16_t> clone_plane(const h266_plane &p) {
  return std::vector<uint16_t>(p.samples, p.samples + (size_t)p.stride * p.height);
}

// apply_sao_clipped, src/sao.rs:389-497
static void apply_sao_clipped(h266_picture *out, const h266_sao_picture *sp, const h266_sao_config *cfg,
                              const uint32_t *col_bd, size_t n_col, const uint32_t *row_bd, size_t n_row) {
  size_t n = (size_t)sp->pic_width_in_ctbs_y * sp->pic_height_in_ctbs_y;
  bool all_off = true;
  for (size_t i = 0; i < n; ++i)
    if (sp->ctbs[i].luma.sao_type_idx != 0 || sp->ctbs[i].cb.sao_type_idx != 0 || sp->ctbs[i].cr.sao_type_idx != 0)
      all_off = false;
  if (all_off) return;
  if (!cfg->luma_used && !cfg->chroma_used) return;
  std::vector<uint16_t> luma_pre, cb_pre, cr_pre;
  if (cfg->luma_used) luma_pre = clone_plane(out->luma);
  bool chroma = cfg->chroma_used && cfg->chroma_format_idc != 0;
  if (chroma) {
    cb_pre = clone_plane(out->cb);
    cr_pre = clone_plane(out->cr);
  }
  int sw, sh;
  chroma_sub(cfg->chroma_format_idc, sw, sh);
  uint32_t ctb = 1u << cfg->ctb_log2_size_y;
  Plane L = mk(out->luma), CB = mk(out->cb), CR = mk(out->cr);
  for (uint32_t ry = 0; ry < sp->pic_height_in_ctbs_y; ++ry)
    for (uint32_t rx = 0; rx < sp->pic_width_in_ctbs_y; ++rx) {
      const h266_sao_ctb_params &p = sp->ctbs[(size_t)ry * sp->pic_width_in_ctbs_y + rx];
      bool has_clip = col_bd != nullptr;
      int cy_[4] = {0, 0, 0, 0}, cc_[4] = {0, 0, 0, 0};
      if (has_clip) {
        span(col_bd, n_col, rx * ctb, (int)out->luma.width, cy_[0], cy_[2]);
        span(row_bd, n_row, ry * ctb, (int)out->luma.height, cy_[1], cy_[3]);
        cc_[0] = cy_[0] / sw;
        cc_[1] = cy_[1] / sh;
        cc_[2] = (cy_[2] + sw - 1) / sw;
        cc_[3] = (cy_[3] + sh - 1) / sh;
      }
      if (cfg->luma_used && p.luma.sao_type_idx != 0)
        apply_sao_ctb(L, luma_pre.data(), has_clip, cy_, rx, ry, ctb, ctb, cfg->bit_depth, p.luma);
      if (chroma) {
        uint32_t nw = ctb / sw, nh = ctb / sh;
        if (p.cb.sao_type_idx != 0) apply_sao_ctb(CB, cb_pre.data(), has_clip, cc_, rx, ry, nw, nh, cfg->bit_depth, p.cb);
        if (p.cr.sao_type_idx != 0) apply_sao_ctb(CR, cr_pre.data(), has_clip, cc_, rx, ry, nw, nh, cfg->bit_depth, p.cr);
      }
    }
}

// ---------------------------------------------------------------------------
// alf.rs
// ---------------------------------------------------------------------------

// resolve_clip_value, src/alf.rs:627-644 (Table 8)
int resolve_clip_value(uint32_t bd, uint8_t clip_idx) {
  static const uint8_t EXP[9][4] = {{8, 5, 3, 1},   {9, 6, 4, 2},    {10, 7, 5, 3},  {11, 8, 6, 4},  {12, 9, 7, 5},
                                    {13, 10, 8, 6}, {14, 11, 9, 7}, {15, 12, 10, 8}, {16, 13, 11, 9}};
  uint32_t row = std::min(std::max(bd, 8u), 16u) - 8;
  return 1 << EXP[row][clip_idx & 3];
}

// transpose_idx_table, src/alf.rs:731-742
const int *transpose_idx_table(int t) {
  static const int T[4][12] = {{0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11},
                               {9, 4, 10, 8, 1, 5, 11, 7, 3, 0, 2, 6},
                               {0, 3, 2, 1, 8, 7, 6, 5, 4, 9, 10, 11},
                               {9, 8, 10, 4, 3, 7, 11, 5, 1, 0, 2, 6}};
  return T[(t >= 1 && t <= 3) ? t : 0];
}

// table_45, src/alf.rs:1117-1130
void table_45(int y, int ctb, bool apply, int out[4]) {
  int a = 7, y1 = 1, y2 = 2, y3 = 3;
  if (apply) {
    if (y == ctb - 5 || y == ctb - 4) { a = 10; y1 = 0; y2 = 0; y3 = 0; }
    else if (y == ctb - 6 || y == ctb - 3) { y1 = 1; y2 = 1; y3 = 1; }
    else if (y == ctb - 7 || y == ctb - 2) { y1 = 1; y2 = 2; y3 = 2; }
  }
  out[0] = a; out[1] = y1; out[2] = y2; out[3] = y3;
}
// table_46, src/alf.rs:1133-1143
void table_46(int y, int h, bool apply, int out[3]) {
  int a = 7, y1 = 1, y2 = 2;
  if (apply) {
    if (y == h - 2 || y == h - 3) { a = 10; y1 = 0; y2 = 0; }
    else if (y == h - 1 || y == h - 4) { y1 = 1; y2 = 1; }
  }
  out[0] = a; out[1] = y1; out[2] = y2;
}
// cc_alf_table_47, src/alf.rs:528-539
void cc_alf_table_47(int y_line, int ctb, bool apply, int out[2]) {
  out[0] = 1; out[1] = 2;
  if (apply) {
    if (y_line == ctb - 5 || y_line == ctb - 4) { out[0] = 0; out[1] = 0; }
    else if (y_line == ctb - 6 || y_line == ctb - 3) { out[0] = 1; out[1] = 1; }
  }
}

// sample, src/alf.rs:1104-1109
static inline int smp(const uint16_t *buf, size_t stride, const int clip[4], int x, int y) {
  int xc = clampi(x, clip[0], clip[2] - 1), yc = clampi(y, clip[1], clip[3] - 1);
  return buf[(size_t)yc * stride + xc];
}

// derive_luma_classification, src/alf.rs:822-1010. Fills (filtIdx, transposeIdx)
// for the (ctb/4)^2 sub-blocks in raster order.
void derive_luma_classification(const uint16_t *pre, size_t stride, int ph, const int clip[4], uint32_t rx,
                                 uint32_t ry, uint32_t ctb_size, uint32_t bd, uint8_t *filt, uint8_t *tr) {
  int x_ctb = (int)(rx * ctb_size), y_ctb = (int)(ry * ctb_size), ctb = (int)ctb_size;
  int sub = (int)ctb_size >> 2;
  bool bottom = y_ctb + ctb >= ph;
  int rem = ph - y_ctb;
  bool carve = !bottom || rem > ctb - 4;
  static const uint8_t VAR_TAB[16] = {0, 1, 2, 2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3, 4};
  static const uint8_t TT[8] = {0, 1, 0, 2, 2, 3, 1, 3};
  for (int sy = 0; sy < sub; ++sy)
    for (int sx = 0; sx < sub; ++sx) {
      int x4 = sx << 2, y4 = sy << 2;
      int min_y = -2, max_y = 5, ac = 2;
      if (y4 == ctb - 8 && carve) { min_y = -2; max_y = 3; ac = 3; }
      else if (y4 == ctb - 4 && carve) { min_y = 0; max_y = 5; ac = 3; }
      int vb = y_ctb + ctb - 4;
      bool has_top = y4 >= ctb - 4;
      bool has_bot = ctb - 4 - y4 > 0 && ctb - 4 - y4 < 5;
      auto pad_y = [&](int cy) {
        int v = cy;
        if (has_top) v = std::max(v, vb);
        if (has_bot) v = std::min(v, vb - 1);
        return v;
      };
      int sh = 0, sv = 0, sd0 = 0, sd1 = 0;
      for (int j = min_y; j <= max_y; ++j)
        for (int i = -2; i <= 5; ++i) {
          if (((i % 2) + 2) % 2 != ((j % 2) + 2) % 2) continue;
          int cx = x_ctb + x4 + i;
          int cy = pad_y(y_ctb + y4 + j), cu = pad_y(y_ctb + y4 + j - 1), cd = pad_y(y_ctb + y4 + j + 1);
          int c2 = smp(pre, stride, clip, cx, cy) * 2;
          sh += absi(c2 - smp(pre, stride, clip, cx - 1, cy) - smp(pre, stride, clip, cx + 1, cy));
          sv += absi(c2 - smp(pre, stride, clip, cx, cu) - smp(pre, stride, clip, cx, cd));
          sd0 += absi(c2 - smp(pre, stride, clip, cx - 1, cu) - smp(pre, stride, clip, cx + 1, cd));
          sd1 += absi(c2 - smp(pre, stride, clip, cx + 1, cu) - smp(pre, stride, clip, cx - 1, cd));
        }
      int hv1, hv0, dir_hv;
      if (sv > sh) { hv1 = sv; hv0 = sh; dir_hv = 1; }
      else { hv1 = sh; hv0 = sv; dir_hv = 3; }
      int d1, d0, dir_d;
      if (sd0 > sd1) { d1 = sd0; d0 = sd1; dir_d = 0; }
      else { d1 = sd1; d0 = sd0; dir_d = 2; }
      bool prefer_d = (int64_t)d1 * hv0 > (int64_t)hv1 * d0;
      int hvd1 = prefer_d ? d1 : hv1, hvd0 = prefer_d ? d0 : hv0;
      int dir1 = prefer_d ? dir_d : dir_hv, dir2 = prefer_d ? dir_hv : dir_d;
      int dir_s = hvd1 * 2 > 9 * hvd0 ? 2 : (hvd1 > 2 * hvd0 ? 1 : 0);
      int64_t prod = (int64_t)(sh + sv) * ac;
      int shifted = (int)clampl(prod >> ((int64_t)bd - 1), 0, 15);
      int fi = VAR_TAB[shifted];
      int ti = TT[dir1 * 2 + (dir2 >> 1)];
      if (dir_s != 0) fi += (((dir1 & 1) << 1) + dir_s) * 5;
      filt[sy * sub + sx] = (uint8_t)fi;
      tr[sy * sub + sx] = (uint8_t)ti;
    }
}

struct LumaSet {
  int coeff[25][12];
  uint8_t clip[25][12];
};

// resolve_luma_filter_set, src/alf.rs:564-595
static bool resolve_luma_filter_set(uint8_t idx, const h266_alf_aps_binding *b, LumaSet &set) {
  if (idx < 16) {
    for (int c = 0; c < 25; ++c) {
      const signed char *row = kAlfFixFiltCoeff[kAlfClassToFiltMap[idx][c]];
      for (int j = 0; j < 12; ++j) {
        set.coeff[c][j] = row[j];
        set.clip[c][j] = 0;
      }
    }
    return true;
  }
  uint32_t slot = (uint32_t)idx - 16;
  if (!b || slot >= b->n_luma_apses || !b->luma_apses[slot]) return false;
  const h266_alf_aps_data *aps = b->luma_apses[slot];
  if (!aps->alf_luma_filter_signal_flag) return false;
  for (int c = 0; c < 25; ++c)
    for (int j = 0; j < 12; ++j) {
      set.coeff[c][j] = aps->luma_coeff[c][j];
      set.clip[c][j] = aps->luma_clip_idx[c][j];
    }
  return true;
}

// apply_alf_luma_ctb, src/alf.rs:652-724
static void apply_alf_luma_ctb(Plane &pl, const uint16_t *pre, const int clip[4], uint32_t rx, uint32_t ry,
                               uint32_t ctb_size, uint32_t bd, const LumaSet &fs, const uint8_t *cf,
                               const uint8_t *ct) {
  size_t x_ctb = (size_t)rx * ctb_size, y_ctb = (size_t)ry * ctb_size;
  size_t stride = pl.stride;
  size_t i_max = std::min<size_t>(ctb_size, (size_t)pl.w > x_ctb ? pl.w - x_ctb : 0);
  size_t j_max = std::min<size_t>(ctb_size, (size_t)pl.h > y_ctb ? pl.h - y_ctb : 0);
  int max_val = (1 << bd) - 1;
  int sub = (int)ctb_size >> 2;
  for (size_t j = 0; j < j_max; ++j)
    for (size_t i = 0; i < i_max; ++i) {
      int xs = (int)(x_ctb + i), ys = (int)(y_ctb + j);
      int fidx = cf[(j >> 2) * sub + (i >> 2)], tidx = ct[(j >> 2) * sub + (i >> 2)];
      const int *f = fs.coeff[fidx];
      const int *idx = transpose_idx_table(tidx);
      int c[12];
      for (int k = 0; k < 12; ++k) c[k] = resolve_clip_value(bd, fs.clip[fidx][k]);
      int t45[4];
      table_45((int)j, (int)ctb_size, true, t45);
      int sh = t45[0], y1 = t45[1], y2 = t45[2], y3 = t45[3];
      int curr = smp(pre, stride, clip, xs, ys);
      auto cl = [&](int k, int dx, int dy) {
        int v = smp(pre, stride, clip, xs + dx, ys + dy) - curr;
        return clampi(v, -c[idx[k]], c[idx[k]]);
      };
      int sum = 0;
      sum += f[idx[0]] * (cl(0, 0, y3) + cl(0, 0, -y3));
      sum += f[idx[1]] * (cl(1, 1, y2) + cl(1, -1, -y2));
      sum += f[idx[2]] * (cl(2, 0, y2) + cl(2, 0, -y2));
      sum += f[idx[3]] * (cl(3, -1, y2) + cl(3, 1, -y2));
      sum += f[idx[4]] * (cl(4, 2, y1) + cl(4, -2, -y1));
      sum += f[idx[5]] * (cl(5, 1, y1) + cl(5, -1, -y1));
      sum += f[idx[6]] * (cl(6, 0, y1) + cl(6, 0, -y1));
      sum += f[idx[7]] * (cl(7, -1, y1) + cl(7, 1, -y1));
      sum += f[idx[8]] * (cl(8, -2, y1) + cl(8, 2, -y1));
      sum += f[idx[9]] * (cl(9, 3, 0) + cl(9, -3, 0));
      sum += f[idx[10]] * (cl(10, 2, 0) + cl(10, -2, 0));
      sum += f[idx[11]] * (cl(11, 1, 0) + cl(11, -1, 0));
      int bias = 1 << (sh - 1);
      int nv = curr + ((sum + bias) >> sh);
      pl.s[(size_t)ys * stride + xs] = (uint16_t)clampi(nv, 0, max_val);
    }
}

// apply_alf_chroma_ctb, src/alf.rs:1014-1065
static void apply_alf_chroma_ctb(Plane &pl, const uint16_t *pre, const int clip[4], uint32_t rx, uint32_t ry,
                                 uint32_t ctb_size, int sw, int sh, uint32_t bd, const int32_t *f,
                                 const uint8_t *clip_idx) {
  size_t w_c = ctb_size / sw, h_c = ctb_size / sh;
  size_t x_ctb = rx * w_c, y_ctb = ry * h_c;
  size_t stride = pl.stride;
  size_t i_max = std::min<size_t>(w_c, (size_t)pl.w > x_ctb ? pl.w - x_ctb : 0);
  size_t j_max = std::min<size_t>(h_c, (size_t)pl.h > y_ctb ? pl.h - y_ctb : 0);
  int max_val = (1 << bd) - 1;
  int c[6];
  for (int k = 0; k < 6; ++k) c[k] = resolve_clip_value(bd, clip_idx[k]);
  for (size_t j = 0; j < j_max; ++j)
    for (size_t i = 0; i < i_max; ++i) {
      int xs = (int)(x_ctb + i), ys = (int)(y_ctb + j);
      int t46[3];
      table_46((int)j, (int)h_c, true, t46);
      int shc = t46[0], y1 = t46[1], y2 = t46[2];
      int curr = smp(pre, stride, clip, xs, ys);
      auto cl = [&](int k, int dx, int dy) {
        int v = smp(pre, stride, clip, xs + dx, ys + dy) - curr;
        return clampi(v, -c[k], c[k]);
      };
      int sum = 0;
      sum += f[0] * (cl(0, 0, y2) + cl(0, 0, -y2));
      sum += f[1] * (cl(1, 1, y1) + cl(1, -1, -y1));
      sum += f[2] * (cl(2, 0, y1) + cl(2, 0, -y1));
      sum += f[3] * (cl(3, -1, y1) + cl(3, 1, -y1));
      sum += f[4] * (cl(4, 2, 0) + cl(4, -2, 0));
      sum += f[5] * (cl(5, 1, 0) + cl(5, -1, 0));
      int bias = 1 << (shc - 1);
      int nv = curr + ((sum + bias) >> shc);
      pl.s[(size_t)ys * stride + xs] = (uint16_t)clampi(nv, 0, max_val);
    }
}

// apply_cc_alf_ctb, src/alf.rs:447-523
static void apply_cc_alf_ctb(Plane &chroma, const uint16_t *luma_pre, size_t luma_stride, int luma_h,
                             const int clip[4], uint32_t rx, uint32_t ry, uint32_t ctb_size, int sw, int sh,
                             uint32_t bd, const int32_t *coeff) {
  size_t w = ctb_size / sw, h = ctb_size / sh;
  size_t x_ctb_c = (rx * ctb_size) / sw, y_ctb_c = (ry * ctb_size) / sh;
  size_t i_max = std::min<size_t>(w, (size_t)chroma.w > x_ctb_c ? chroma.w - x_ctb_c : 0);
  size_t j_max = std::min<size_t>(h, (size_t)chroma.h > y_ctb_c ? chroma.h - y_ctb_c : 0);
  int max_val = (1 << bd) - 1;
  int half = 1 << (bd - 1);
  int ph = luma_h;
  for (size_t y = 0; y < j_max; ++y)
    for (size_t x = 0; x < i_max; ++x) {
      int xl = (int)(x_ctb_c + x) * sw, yl = (int)(y_ctb_c + y) * sh;
      int y_line = (int)y * sh;
      bool apply_lbb = !(yl + (int)ctb_size >= ph && (ph - (int)y_ctb_c * sh) <= (int)ctb_size - 4);
      int t47[2];
      cc_alf_table_47(y_line, (int)ctb_size, apply_lbb, t47);
      int yp1 = t47[0], yp2 = t47[1];
      size_t at = (y_ctb_c + y) * chroma.stride + (x_ctb_c + x);
      int curr = chroma.s[at];
      int centre = smp(luma_pre, luma_stride, clip, xl, yl);
      int sum = 0;
      sum += coeff[0] * (smp(luma_pre, luma_stride, clip, xl, yl - yp1) - centre);
      sum += coeff[1] * (smp(luma_pre, luma_stride, clip, xl - 1, yl) - centre);
      sum += coeff[2] * (smp(luma_pre, luma_stride, clip, xl + 1, yl) - centre);
      sum += coeff[3] * (smp(luma_pre, luma_stride, clip, xl - 1, yl + yp1) - centre);
      sum += coeff[4] * (smp(luma_pre, luma_stride, clip, xl, yl + yp1) - centre);
      sum += coeff[5] * (smp(luma_pre, luma_stride, clip, xl + 1, yl + yp1) - centre);
      sum += coeff[6] * (smp(luma_pre, luma_stride, clip, xl, yl + yp2) - centre);
      int scaled = clampi((sum + 64) >> 7, -half, half - 1);
      bool suppress = sh == 1 && (y_line == (int)ctb_size - 3 || y_line == (int)ctb_size - 4);
      int nv = suppress ? curr : curr + scaled;
      chroma.s[at] = (uint16_t)clampi(nv, 0, max_val);
    }
}

// clip_rect_for_ctb, src/alf.rs:1071-1095
static void clip_rect_for_ctb(uint32_t rx, uint32_t ry, uint32_t ctb, int pw, int ph, const uint32_t *col_bd,
                              size_t n_col, const uint32_t *row_bd, size_t n_row, int r[4]) {
  if (!col_bd) {
    r[0] = 0; r[1] = 0; r[2] = pw; r[3] = ph;
    return;
  }
  span(col_bd, n_col, rx * ctb, pw, r[0], r[2]);
  span(row_bd, n_row, ry * ctb, ph, r[1], r[3]);
}

// apply_alf_clipped, src/alf.rs:235-434
static void apply_alf_clipped(h266_picture *out, const h266_alf_picture *ap, const h266_alf_config *cfg,
                              const h266_alf_aps_binding *b, const uint32_t *col_bd, size_t n_col,
                              const uint32_t *row_bd, size_t n_row) {
  if (!cfg->alf_enabled) return;
  size_t n = (size_t)ap->pic_width_in_ctbs_y * ap->pic_height_in_ctbs_y;
  bool all_off = true;
  for (size_t i = 0; i < n; ++i) {
    const h266_alf_ctb &c = ap->ctbs[i];
    if (c.luma_on || c.cb_on || c.cr_on || c.cc_cb_idc != 0 || c.cc_cr_idc != 0) all_off = false;
  }
  if (all_off) return;
  uint32_t ctb = 1u << cfg->ctb_log2_size_y;
  int sw, sh;
  chroma_sub(cfg->chroma_format_idc, sw, sh);
  std::vector<uint16_t> luma_pre = clone_plane(out->luma), cb_pre, cr_pre;
  if (cfg->chroma_format_idc != 0) {
    cb_pre = clone_plane(out->cb);
    cr_pre = clone_plane(out->cr);
  }
  int lw = (int)out->luma.width, lh = (int)out->luma.height;
  Plane L = mk(out->luma), CB = mk(out->cb), CR = mk(out->cr);
  int sub = (int)ctb >> 2;
  std::vector<uint8_t> cf((size_t)sub * sub), ct((size_t)sub * sub);
  for (uint32_t ry = 0; ry < ap->pic_height_in_ctbs_y; ++ry)
    for (uint32_t rx = 0; rx < ap->pic_width_in_ctbs_y; ++rx) {
      const h266_alf_ctb &p = ap->ctbs[(size_t)ry * ap->pic_width_in_ctbs_y + rx];
      int fy[4];
      clip_rect_for_ctb(rx, ry, ctb, lw, lh, col_bd, n_col, row_bd, n_row, fy);
      int fc[4] = {fy[0] / sw, fy[1] / sh, (fy[2] + sw - 1) / sw, (fy[3] + sh - 1) / sh};
      if (p.luma_on) {
        LumaSet fs;
        if (resolve_luma_filter_set(p.luma_filt_set_idx, b, fs)) {
          derive_luma_classification(luma_pre.data(), out->luma.stride, lh, fy, rx, ry, ctb, cfg->bit_depth,
                                     cf.data(), ct.data());
          apply_alf_luma_ctb(L, luma_pre.data(), fy, rx, ry, ctb, cfg->bit_depth, fs, cf.data(), ct.data());
        }
      }
      if (cfg->chroma_format_idc != 0) {
        const h266_alf_aps_data *aps = b ? b->chroma_aps : nullptr;
        auto chroma_one = [&](bool on, uint8_t alt, Plane &pl, const std::vector<uint16_t> &pre) {
          if (!on || !aps) return;
          if (!aps->alf_chroma_filter_signal_flag) return;  // resolve_chroma_filter src/alf.rs:603
          if (alt >= aps->n_chroma_filters) return;          // src/alf.rs:606
          apply_alf_chroma_ctb(pl, pre.data(), fc, rx, ry, ctb, sw, sh, cfg->bit_depth, aps->chroma_coeff[alt],
                               aps->chroma_clip_idx[alt]);
        };
        chroma_one(cfg->cb_enabled && p.cb_on, p.cb_alt_idx, CB, cb_pre);
        chroma_one(cfg->cr_enabled && p.cr_on, p.cr_alt_idx, CR, cr_pre);
      }
    }
  if (cfg->chroma_format_idc != 0) {
    for (uint32_t ry = 0; ry < ap->pic_height_in_ctbs_y; ++ry)
      for (uint32_t rx = 0; rx < ap->pic_width_in_ctbs_y; ++rx) {
        const h266_alf_ctb &p = ap->ctbs[(size_t)ry * ap->pic_width_in_ctbs_y + rx];
        int fy[4];
        clip_rect_for_ctb(rx, ry, ctb, lw, lh, col_bd, n_col, row_bd, n_row, fy);
        if (cfg->cc_cb_enabled && p.cc_cb_idc != 0 && b && b->cc_cb_aps) {
          uint32_t fi = p.cc_cb_idc - 1;
          if (fi < b->cc_cb_aps->n_cc_cb_filters)
            apply_cc_alf_ctb(CB, luma_pre.data(), out->luma.stride, lh, fy, rx, ry, ctb, sw, sh, cfg->bit_depth,
                             b->cc_cb_aps->cc_cb_coeff[fi]);
        }
        if (cfg->cc_cr_enabled && p.cc_cr_idc != 0 && b && b->cc_cr_aps) {
          uint32_t fi = p.cc_cr_idc - 1;
          if (fi < b->cc_cr_aps->n_cc_cr_filters)
            apply_cc_alf_ctb(CR, luma_pre.data(), out->luma.stride, lh, fy, rx, ry, ctb, sw, sh, cfg->bit_depth,
                             b->cc_cr_aps->cc_cr_coeff[fi]);
        }
      }
  }
}

// ---------------------------------------------------------------------------
// lmcs.rs
// ---------------------------------------------------------------------------

// derive_lmcs, src/lmcs.rs:302-404. Returns 0 on success, -3 where the crate returns Err.
int derive_lmcs(const h266_lmcs_data *d, uint32_t bd, h266_lmcs_derived *o) {
  if (bd < 8 || bd > 16) return -3;
  std::memset(o, 0, sizeof *o);
  if (d->lmcs_delta_max_bin_idx > 15) return -3;
  uint32_t org_cw = (1u << bd) / 16, log2_org = bd - 4;
  uint32_t band_lo = org_cw >> 3, band_hi = (org_cw << 3) - 1;
  uint32_t mn = d->lmcs_min_bin_idx, mx = 15u - d->lmcs_delta_max_bin_idx;
  for (uint32_t i = mn; i <= mx && i < 16; ++i) {
    int64_t delta = (int64_t)d->lmcs_delta_abs_cw[i] * (d->lmcs_delta_sign_cw_flag[i] ? -1 : 1);
    int64_t v = (int64_t)org_cw + delta;
    if (v < (int64_t)band_lo || v > (int64_t)band_hi) return -3;
    o->lmcs_cw[i] = (uint32_t)v;
  }
  uint32_t total = 0;
  for (int i = 0; i < 16; ++i) total += o->lmcs_cw[i];
  if (total > (1u << bd) - 1) return -3;
  for (uint32_t i = 0; i < 16; ++i) o->input_pivot[i] = i * org_cw;
  for (int i = 0; i < 16; ++i) {
    o->lmcs_pivot[i + 1] = o->lmcs_pivot[i] + o->lmcs_cw[i];
    o->scale_coeff[i] = (o->lmcs_cw[i] * (1u << 11) + (1u << (log2_org - 1))) >> log2_org;
    o->inv_scale_coeff[i] = o->lmcs_cw[i] ? (org_cw * (1u << 11)) / o->lmcs_cw[i] : 0;
  }
  uint32_t shift = bd - 5;
  for (uint32_t i = mn; i <= mx && i < 16; ++i)
    if (o->lmcs_pivot[i] % (1u << shift) != 0 && (o->lmcs_pivot[i] >> shift) == (o->lmcs_pivot[i + 1] >> shift))
      return -3;
  int32_t crs = (int32_t)d->lmcs_delta_abs_crs * (d->lmcs_delta_sign_crs_flag ? -1 : 1);
  for (int i = 0; i < 16; ++i) {
    if (o->lmcs_cw[i] == 0) {
      o->chroma_scale_coeff[i] = 1u << 11;
    } else {
      int64_t joint = (int64_t)o->lmcs_cw[i] + crs;
      if (joint < (int64_t)band_lo || joint > (int64_t)band_hi) return -3;
      o->chroma_scale_coeff[i] = org_cw * (1u << 11) / (uint32_t)joint;
    }
  }
  o->bit_depth = bd;
  o->org_cw = org_cw;
  o->lmcs_delta_crs = crs;
  return 0;
}

// LmcsDerived::idx_y_inv, src/lmcs.rs:209-220
uint32_t idx_y_inv(const h266_lmcs_derived *l, uint32_t s, uint32_t mn, uint32_t mx) {
  uint32_t idx = mn;
  while (idx <= mx) {
    if (s < l->lmcs_pivot[idx + 1]) break;
    idx += 1;
  }
  return std::min(idx, 15u);
}
// LmcsDerived::inverse_map_luma_sample, src/lmcs.rs:230-238
uint32_t inverse_map(const h266_lmcs_derived *l, uint32_t s, uint32_t idx) {
  int64_t prod = (int64_t)l->inv_scale_coeff[idx] * ((int64_t)s - (int64_t)l->lmcs_pivot[idx]) + (1 << 10);
  int64_t inv = (int64_t)l->input_pivot[idx] + (prod >> 11);
  return (uint32_t)clampl(inv, 0, (1LL << l->bit_depth) - 1);
}
// LmcsDerived::forward_map_luma_sample, src/lmcs.rs:186-194 (round-trip tests only)
int64_t forward_map(const h266_lmcs_derived *l, uint32_t s) {
  uint32_t idx = s >> (l->bit_depth - 4);
  int64_t prod = (int64_t)l->scale_coeff[idx] * ((int64_t)s - (int64_t)l->input_pivot[idx]) + (1 << 10);
  return (int64_t)l->lmcs_pivot[idx] + (prod >> 11);
}
// LmcsDerived::scale_chroma_residual_sample, src/lmcs.rs:257-279 (derivation tests only)
uint32_t scale_chroma_residual(const h266_lmcs_derived *l, int64_t pred, int64_t res, uint32_t var_scale) {
  int64_t lo = -(1LL << l->bit_depth), hi = (1LL << l->bit_depth) - 1;
  int64_t r = clampl(res, lo, hi);
  int64_t scaled = 0;
  if (r != 0) {
    uint64_t mag = ((uint64_t)(r < 0 ? -r : r) * var_scale + (1u << 10)) >> 11;
    scaled = r < 0 ? -(int64_t)mag : (int64_t)mag;
  }
  return (uint32_t)clampl(pred + scaled, 0, (1LL << l->bit_depth) - 1);
}

// The driver loop src/ctu.rs:11837-11851.
static void lmcs_inverse_plane(h266_plane &p, const h266_lmcs_derived *l, uint32_t mn, uint32_t mx) {
  for (uint32_t r = 0; r < p.height; ++r)
    for (uint32_t c = 0; c < p.width; ++c) {
      uint16_t &s = p.samples[(size_t)r * p.stride + c];
      uint32_t iy = idx_y_inv(l, s, mn, mx);
      s = (uint16_t)inverse_map(l, s, iy);
    }
}

// apply_in_loop_filters_with_alf after its gate lists, src/ctu.rs:11822-12065.
static void chain(h266_picture *pic, const h266_in_loop_filter_args *a) {
  if (a->lmcs) lmcs_inverse_plane(pic->luma, a->lmcs, a->lmcs_min_bin_idx, a->lmcs_max_bin_idx);
  apply_deblocking_clipped(pic, a->cus, a->n_cus, a->chroma_cus, a->n_chroma_cus, a->mv_grid, &a->deblock,
                           a->chroma_format_idc, a->no_filter_cols, a->n_no_filter_cols, a->no_filter_rows,
                           a->n_no_filter_rows, nullptr, true);
  if (a->sao)
    apply_sao_clipped(pic, a->sao, &a->sao_cfg, a->clip_cols, a->n_clip_cols, a->clip_rows, a->n_clip_rows);
  if (a->alf)
    apply_alf_clipped(pic, a->alf, &a->alf_cfg, a->alf_binding, a->clip_cols, a->n_clip_cols, a->clip_rows,
                      a->n_clip_rows);
}

// CtuWalker::lmcs_forward_map_luma_rect (src/ctu.rs:1701-1727), one call per
// rectangle in list order.  Returns false where the crate would index past its
// 16 bins (a sample above 2^BitDepth - 1), leaving the rest unmapped.
static bool lmcs_forward_map_rects(h266_plane &pl, const h266_lmcs_derived *l, const h266_rect *rects, size_t n) {
  const int64_t hi = ((int64_t)1 << l->bit_depth) - 1;
  for (size_t r = 0; r < n; ++r) {
    const uint64_t y1 = std::min<uint64_t>((uint64_t)rects[r].y + rects[r].h, pl.height);
    const uint64_t x1 = std::min<uint64_t>((uint64_t)rects[r].x + rects[r].w, pl.width);
    for (uint64_t row = rects[r].y; row < y1; ++row)
      for (uint64_t col = rects[r].x; col < x1; ++col) {
        uint16_t &v = pl.samples[row * pl.stride + col];
        if ((v >> (l->bit_depth - 4)) > 15) return false;
        v = (uint16_t)clampl(forward_map(l, v), 0, hi);
      }
  }
  return true;
}

// CtuWalker::lmcs_chroma_var_scale_for_cu (src/ctu.rs:1752-1815) from
// (xCuCb, yCuCb) and the neighbour availability on.
static uint32_t lmcs_chroma_var_scale(const h266_plane &luma, const h266_lmcs_derived *l, uint32_t mn, uint32_t mx,
                                      uint32_t size_y, const h266_lmcs_cvs_block &b) {
  const bool avail_l = b.x_cu_cb > 0 && b.avail_l, avail_t = b.y_cu_cb > 0 && b.avail_t;
  uint64_t sum = 0, cnt = 0;
  if (avail_l) {
    for (uint32_t i = 0; i < size_y; ++i) {
      const uint64_t yy = std::min<uint64_t>((uint64_t)b.y_cu_cb + i, luma.height - 1);
      sum += luma.samples[yy * luma.stride + (b.x_cu_cb - 1)];
    }
    cnt += size_y;
  }
  if (avail_t) {
    for (uint32_t i = 0; i < size_y; ++i) {
      const uint64_t xx = std::min<uint64_t>((uint64_t)b.x_cu_cb + i, luma.width - 1);
      sum += luma.samples[(uint64_t)(b.y_cu_cb - 1) * luma.stride + xx];
    }
    cnt += size_y;
  }
  uint32_t avg;
  if (cnt > 0) {
    int tz = 0;
    while (!((cnt >> tz) & 1)) ++tz;
    avg = (uint32_t)((sum + (cnt >> 1)) >> tz);
  } else {
    avg = 1u << (l->bit_depth - 1);
  }
  return l->chroma_scale_coeff[idx_y_inv(l, avg, mn, mx)];
}

// The inter chroma residual add (src/ctu.rs:9912-9945) with the optional
// lmcs_scale_chroma_residuals fold (src/ctu.rs:734-742).
static void add_chroma_residual(h266_picture *pic, uint32_t bd, const int32_t *res, const h266_chroma_res_block &b) {
  h266_plane &pl = b.plane == 1 ? pic->cb : pic->cr;
  const int64_t lo = -((int64_t)1 << bd), hi = ((int64_t)1 << bd) - 1;
  for (uint32_t row = 0; row < b.h; ++row)
    for (uint32_t col = 0; col < b.w; ++col) {
      int64_t r = res[b.res_offset + (uint64_t)row * b.w + col];
      if (b.var_scale != H266_NO_VAR_SCALE) {
        const int64_t v = clampl(r, lo, hi);
        const int64_t mag = (int64_t)(((uint64_t)(v < 0 ? -v : v) * b.var_scale + 1024) >> 11);
        r = v < 0 ? -mag : mag;
      }
      uint16_t &s = pl.samples[(uint64_t)(b.y + row) * pl.stride + b.x + col];
      s = (uint16_t)clampl((int64_t)s + r, 0, hi);
    }
}

// The cropped planar dump of examples/decode_dump.rs:24-40 (and the per-plane
// serialisation hashed by tests/jvet_conformance.rs:402-427): luma, then Cb and
// Cr with the crop halved when chroma_format_idc != 0; one byte per sample
// (`v as u8`) for BitDepth <= 8, else two bytes little-endian.
static uint64_t output_convert(const h266_picture *pic, const h266_crop_window &c, uint32_t cfi, uint32_t bd,
                               uint8_t *out) {
  const bool wide = bd > 8;
  struct P { const h266_plane *p; uint32_t x0, y0, w, h; };
  P planes[3] = {{&pic->luma, c.left, c.top, c.width, c.height},
                 {&pic->cb, c.left / 2, c.top / 2, c.width / 2, c.height / 2},
                 {&pic->cr, c.left / 2, c.top / 2, c.width / 2, c.height / 2}};
  uint64_t o = 0;
  for (int i = 0; i < (cfi != 0 ? 3 : 1); ++i) {
    const P &q = planes[i];
    for (uint64_t y = q.y0; y < (uint64_t)q.y0 + q.h; ++y)
      for (uint64_t x = q.x0; x < (uint64_t)q.x0 + q.w; ++x) {
        const uint16_t v = q.p->samples[y * q.p->stride + x];
        if (wide) {
          out[o++] = (uint8_t)(v & 0xFF);
          out[o++] = (uint8_t)(v >> 8);
        } else {
          out[o++] = (uint8_t)v;
        }
      }
  }
  return o;
}

// ---- encoder SAO decision (src/sao_enc.rs:44-487)
static bool pget(const h266_plane &p, int64_t x, int64_t y, uint16_t &v) {  // PicturePlane::get
  if (x < 0 || y < 0 || x >= (int64_t)p.width || y >= (int64_t)p.height) return false;
  v = p.samples[(size_t)y * p.stride + (size_t)x];
  return true;
}

// derive_offset_val, src/sao.rs:356-365
static void sao_offsets(h266_sao_ctb &c, const uint32_t abs_[4], const uint32_t sign[4], uint32_t bd) {
  const int shift = (int)bd - (int)std::min<uint32_t>(bd, 10);
  c.offset_val[0] = 0;
  for (int i = 0; i < 4; ++i) c.offset_val[i + 1] = (1 - 2 * (int)(sign[i] & 1)) * (int)(abs_[i] << shift);
}

// try_band_offset, src/sao_enc.rs:77-171
static bool try_band_offset(const h266_plane &src, const h266_plane &rec, size_t cx, size_t cy, size_t cw, size_t ch,
                            uint32_t bd, h266_sao_ctb &out) {
  int64_t cnt[32] = {0}, dif[32] = {0};
  const uint32_t shift = bd - 5;
  const size_t xe = std::min<size_t>(cx + cw, rec.width), ye = std::min<size_t>(cy + ch, rec.height);
  for (size_t y = cy; y < ye; ++y)
    for (size_t x = cx; x < xe; ++x) {
      uint16_t r, s;
      if (pget(rec, x, y, r) && pget(src, x, y, s)) {
        cnt[r >> shift] += 1;
        dif[r >> shift] += (int64_t)s - r;
      }
    }
  int64_t best_delta = 0;
  int best_start = 0, best_off[4] = {0, 0, 0, 0};
  for (int start = 0; start < 28; ++start) {
    int64_t delta = 0;
    int off[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; ++i) {
      const int b = start + i;
      if (cnt[b] > 0) {
        const int64_t cmax = ((int64_t)1 << (std::min<uint32_t>(bd, 10) - 5)) - 1;
        const int64_t opt = (dif[b] + cnt[b] / 2) / cnt[b];
        off[i] = (int)clampl(opt, -cmax, cmax);
        delta -= dif[b] * off[i];
      }
    }
    if (delta < best_delta) {
      best_delta = delta;
      best_start = start;
      std::memcpy(best_off, off, sizeof off);
    }
  }
  if (best_delta >= 0) return false;
  uint32_t a[4], sg[4];
  for (int i = 0; i < 4; ++i) {
    a[i] = (uint32_t)(best_off[i] < 0 ? -best_off[i] : best_off[i]);
    sg[i] = best_off[i] < 0 ? 1 : 0;
  }
  out = h266_sao_ctb{};
  out.sao_type_idx = 1;
  out.band_position = (uint8_t)(best_start & 31);
  sao_offsets(out, a, sg, bd);
  return true;
}

// eo_category, src/sao_enc.rs:349-373
static int eo_category(int r, int n0, int n1) {
  const int s = (r > n0 ? 1 : (r < n0 ? -1 : 0)) + (r > n1 ? 1 : (r < n1 ? -1 : 0));
  switch (s) {
    case 2: return 4;
    case 1: return 3;
    case -1: return 2;
    case -2: return 1;
    default: return 0;
  }
}

// try_edge_offset_class, src/sao_enc.rs:211-284 (the delta uses |diff|, as there)
static void try_edge_offset_class(const h266_plane &src, const h266_plane &rec, size_t cx, size_t cy, size_t cw,
                                  size_t ch, uint32_t bd, int cls, h266_sao_ctb &out, int64_t &delta) {
  static const int kDirs[4][4] = {{-1, 0, 1, 0}, {0, -1, 0, 1}, {-1, -1, 1, 1}, {1, -1, -1, 1}};
  const int *d = kDirs[cls];
  int64_t cnt[5] = {0}, dif[5] = {0};
  const size_t xe = std::min<size_t>(cx + cw, rec.width), ye = std::min<size_t>(cy + ch, rec.height);
  for (size_t y = cy; y < ye; ++y)
    for (size_t x = cx; x < xe; ++x) {
      uint16_t r, a, b, s;
      if (!pget(rec, x, y, r)) continue;
      if (!pget(rec, (int64_t)x + d[0], (int64_t)y + d[1], a) || !pget(rec, (int64_t)x + d[2], (int64_t)y + d[3], b))
        continue;
      const int cat = eo_category(r, a, b);
      if (pget(src, x, y, s)) {
        cnt[cat] += 1;
        dif[cat] += (int64_t)s - r;
      }
    }
  uint32_t off[4] = {0, 0, 0, 0};
  delta = 0;
  for (int i = 0; i < 4; ++i) {
    const int cat = i + 1;
    if (cnt[cat] > 0) {
      const int64_t ad = dif[cat] < 0 ? -dif[cat] : dif[cat];
      off[i] = (uint32_t)clampl((ad + cnt[cat] / 2) / cnt[cat], 0, 7);
      delta -= ad * (int64_t)off[i];
    }
  }
  static const uint32_t kSign[4] = {0, 0, 1, 1};  // SaoCtb::edge_offset, src/sao.rs:169-180
  out = h266_sao_ctb{};
  out.sao_type_idx = 2;
  out.eo_class = (uint8_t)cls;
  sao_offsets(out, off, kSign, bd);
}

// sao_decide_ctb, src/sao_enc.rs:44-70 (with try_best_edge_offset, :175-209)
static h266_sao_ctb sao_decide_ctb(const h266_plane &src, const h266_plane &rec, size_t cx, size_t cy, size_t cw,
                                   size_t ch, uint32_t bd) {
  h266_sao_ctb bo{}, eo{}, t{};
  const bool has_bo = try_band_offset(src, rec, cx, cy, cw, ch, bd, bo);
  int64_t best = 0, delta;
  bool has_eo = false;
  for (int c = 0; c < 4; ++c) {
    try_edge_offset_class(src, rec, cx, cy, cw, ch, bd, c, t, delta);
    if (delta < best) {
      best = delta;
      eo = t;
      has_eo = true;
    }
  }
  if (has_eo) return eo;
  if (has_bo) return bo;
  return h266_sao_ctb{};
}

// sao_decide_ctb_constrained, src/sao_enc.rs:286-347
static h266_sao_ctb sao_decide_ctb_constrained(const h266_plane &src, const h266_plane &rec, size_t cx, size_t cy,
                                               size_t cw, size_t ch, uint32_t bd, const h266_sao_ctb &shared) {
  h266_sao_ctb out{};
  if (shared.sao_type_idx == 1) {
    if (!try_band_offset(src, rec, cx, cy, cw, ch, bd, out)) {
      out = h266_sao_ctb{};
      out.sao_type_idx = 1;
    }
  } else if (shared.sao_type_idx == 2) {
    int64_t delta;
    try_edge_offset_class(src, rec, cx, cy, cw, ch, bd, shared.eo_class, out, delta);
    if (delta >= 0) {
      out = h266_sao_ctb{};
      out.sao_type_idx = 2;
      out.eo_class = shared.eo_class;
    }
  }
  return out;
}

// sao_decide_picture, src/sao_enc.rs:385-487
static void sao_decide_picture(const h266_picture *src, const h266_picture *rec, uint32_t log2, uint32_t bd,
                               bool luma_on, bool chroma_on, h266_sao_ctb_params *out) {
  const size_t ctb = (size_t)1 << log2, pw = rec->luma.width, ph = rec->luma.height;
  const size_t wc = (pw + ctb - 1) / ctb, hc = (ph + ctb - 1) / ctb;
  for (size_t ry = 0; ry < hc; ++ry)
    for (size_t rx = 0; rx < wc; ++rx) {
      const size_t cx = rx * ctb, cy = ry * ctb, cw = std::min(ctb, pw - cx), ch = std::min(ctb, ph - cy);
      h266_sao_ctb_params &p = out[ry * wc + rx];
      p = h266_sao_ctb_params{};
      if (luma_on) p.luma = sao_decide_ctb(src->luma, rec->luma, cx, cy, cw, ch, bd);
      const size_t x2 = cx / 2, y2 = cy / 2, w2 = cw / 2, h2 = ch / 2;
      if (chroma_on && w2 > 0 && h2 > 0) {
        p.cb = sao_decide_ctb(src->cb, rec->cb, x2, y2, w2, h2, bd);
        p.cr = sao_decide_ctb_constrained(src->cr, rec->cr, x2, y2, w2, h2, bd, p.cb);
      }
    }
}

// ctb_sse_y, src/alf_enc.rs:79-105: SSE over the CTB rectangle inside both planes.
static uint64_t ctb_sse_y(const h266_plane &src, const h266_plane &rec, size_t x0, size_t y0, size_t w, size_t h) {
  uint64_t sse = 0;
  for (size_t y = 0; y < h; ++y) {
    const size_t yi = y0 + y;
    if (yi >= src.height || yi >= rec.height) break;
    for (size_t x = 0; x < w; ++x) {
      const size_t xi = x0 + x;
      if (xi >= src.width || xi >= rec.width) break;
      const int64_t d = (int64_t)src.samples[yi * src.stride + xi] - (int64_t)rec.samples[yi * rec.stride + xi];
      sse += (uint64_t)(d * d);
    }
  }
  return sse;
}

// alf_decide_and_apply_clipped (src/alf_enc.rs:185-322) when `aps` is NULL,
// alf_decide_and_apply_with_aps_clipped (src/alf_enc.rs:352-528) otherwise:
// trials 0..15 are the fixed sets (every CTB on), trial 16 the APS set
// (luma_filt_set_idx 16, APS slot 0); per CTB the lowest SSE_Y among
// {off, trial 0, ...} wins (strict <, so earlier options win ties) and its
// luma samples are copied into `rec`.  `decisions` receives the returned
// AlfPicture; `sse` (optional) the per-CTB table [off, trial 0, ...].
static void alf_decide_and_apply(const h266_picture *src, h266_picture *rec, const h266_alf_aps_data *aps,
                                 uint32_t log2, uint32_t bd, uint32_t cfi, const uint32_t *cols, size_t n_cols,
                                 const uint32_t *rows, size_t n_rows, h266_alf_ctb *decisions, uint64_t *sse) {
  const uint32_t ctb = 1u << log2;
  const uint32_t wc = (rec->luma.width + ctb - 1) / ctb, hc = (rec->luma.height + ctb - 1) / ctb;
  const size_t n = (size_t)wc * hc;
  const size_t trials = aps ? 17 : 16;
  std::vector<uint64_t> pre(n);
  for (uint32_t ry = 0; ry < hc; ++ry)
    for (uint32_t rx = 0; rx < wc; ++rx)
      pre[(size_t)ry * wc + rx] = ctb_sse_y(src->luma, rec->luma, (size_t)rx * ctb, (size_t)ry * ctb, ctb, ctb);
  h266_alf_config cfg{};
  cfg.alf_enabled = 1;
  cfg.bit_depth = bd;
  cfg.ctb_log2_size_y = log2;
  cfg.chroma_format_idc = cfi;
  const h266_alf_aps_data *slot[1] = {aps};
  h266_alf_aps_binding binding{};
  if (aps) {
    binding.luma_apses = slot;
    binding.n_luma_apses = 1;
  }
  const size_t lum = (size_t)rec->luma.stride * rec->luma.height;
  std::vector<uint64_t> per(n * trials);
  std::vector<std::vector<uint16_t>> per_luma(trials);
  std::vector<h266_alf_ctb> trial(n);
  for (size_t t = 0; t < trials; ++t) {
    std::vector<uint16_t> y(rec->luma.samples, rec->luma.samples + lum);  // rec.clone() (luma; chroma is untouched)
    h266_picture pic = *rec;
    pic.luma.samples = y.data();
    pic.cb.width = pic.cb.height = 0;
    pic.cr.width = pic.cr.height = 0;
    for (size_t i = 0; i < n; ++i) {
      trial[i] = h266_alf_ctb{};
      trial[i].luma_on = 1;
      trial[i].luma_filt_set_idx = (uint8_t)(t < 16 ? t : 16);
    }
    h266_alf_picture ap{wc, hc, trial.data()};
    apply_alf_clipped(&pic, &ap, &cfg, t < 16 ? nullptr : &binding, cols, n_cols, rows, n_rows);
    for (uint32_t ry = 0; ry < hc; ++ry)
      for (uint32_t rx = 0; rx < wc; ++rx)
        per[((size_t)ry * wc + rx) * trials + t] =
            ctb_sse_y(src->luma, pic.luma, (size_t)rx * ctb, (size_t)ry * ctb, ctb, ctb);
    per_luma[t] = std::move(y);
  }
  const size_t st = rec->luma.stride;
  for (uint32_t ry = 0; ry < hc; ++ry)
    for (uint32_t rx = 0; rx < wc; ++rx) {
      const size_t idx = (size_t)ry * wc + rx;
      uint64_t best = pre[idx];
      int pick = -1;
      for (size_t t = 0; t < trials; ++t)
        if (per[idx * trials + t] < best) {
          best = per[idx * trials + t];
          pick = (int)t;
        }
      decisions[idx] = h266_alf_ctb{};
      if (sse) {
        sse[idx * (trials + 1)] = pre[idx];
        for (size_t t = 0; t < trials; ++t) sse[idx * (trials + 1) + 1 + t] = per[idx * trials + t];
      }
      if (pick < 0) continue;
      const size_t x0 = (size_t)rx * ctb, y0 = (size_t)ry * ctb;
      const size_t w = std::min<size_t>(ctb, rec->luma.width > x0 ? rec->luma.width - x0 : 0);
      const size_t h = std::min<size_t>(ctb, rec->luma.height > y0 ? rec->luma.height - y0 : 0);
      for (size_t y = 0; y < h; ++y)
        std::memcpy(rec->luma.samples + (y0 + y) * st + x0, per_luma[pick].data() + (y0 + y) * st + x0, w * 2);
      decisions[idx].luma_on = 1;
      decisions[idx].luma_filt_set_idx = (uint8_t)(pick < 16 ? pick : 16);
    }
}

// chroma_independent_bit_cost, src/sao_enc.rs:670-696
static int64_t sao_chroma_bits(const h266_sao_ctb_params &p) {
  int64_t bits = 1;
  for (const h266_sao_ctb *c : {&p.cb, &p.cr}) bits += c->sao_type_idx == 0 ? 1 : (c->sao_type_idx == 1 ? 16 : 10);
  return bits;
}

// chroma_ctb_sse_with, src/sao_enc.rs:698-749: SAO of one CTB with the given
// chroma parameters on a copy of the pre-SAO picture, Cb + Cr SSE over the
// CTB's chroma region (Cb's extent for both planes, as there).
static uint64_t chroma_ctb_sse_with(const h266_picture *src, const h266_picture *pre, uint32_t rx, uint32_t ry,
                                    size_t chr_ctb, uint32_t bd, const h266_sao_ctb &cb, const h266_sao_ctb &cr) {
  std::vector<uint16_t> L = clone_plane(pre->luma), B = clone_plane(pre->cb), Cr = clone_plane(pre->cr);
  h266_picture tmp = *pre;
  tmp.luma.samples = L.data();
  tmp.cb.samples = B.data();
  tmp.cr.samples = Cr.data();
  std::vector<h266_sao_ctb_params> one((size_t)(rx + 1) * (ry + 1));
  one[(size_t)ry * (rx + 1) + rx].cb = cb;
  one[(size_t)ry * (rx + 1) + rx].cr = cr;
  const h266_sao_picture sp{rx + 1, ry + 1, one.data()};
  uint32_t log2 = 0;
  while (((size_t)1 << log2) < chr_ctb * 2) ++log2;
  const h266_sao_config cfg{0, 1, bd, log2, 1};
  apply_sao_clipped(&tmp, &sp, &cfg, nullptr, 0, nullptr, 0);
  const size_t cx = (size_t)rx * chr_ctb, cy = (size_t)ry * chr_ctb;
  const size_t cw = std::min(chr_ctb, tmp.cb.width > cx ? tmp.cb.width - cx : 0);
  const size_t ch = std::min(chr_ctb, tmp.cb.height > cy ? tmp.cb.height - cy : 0);
  uint64_t sse = 0;
  for (size_t y = 0; y < ch; ++y)
    for (size_t x = 0; x < cw; ++x) {
      const int64_t dcb = (int64_t)src->cb.samples[(cy + y) * src->cb.stride + cx + x] -
                          (int64_t)tmp.cb.samples[(cy + y) * tmp.cb.stride + cx + x];
      const int64_t dcr = (int64_t)src->cr.samples[(cy + y) * src->cr.stride + cx + x] -
                          (int64_t)tmp.cr.samples[(cy + y) * tmp.cr.stride + cx + x];
      sse += (uint64_t)(dcb * dcb + dcr * dcr);
    }
  return sse;
}

// apply_chroma_sao_merge, src/sao_enc.rs:500-668: raster order; per CTB the
// lowest cost (SSE + 8 * bits) among independent, merge-left (1 bit) and
// merge-above (2 bits), strict < in that order; map: 0 independent, 1 left,
// 2 above.
static void sao_chroma_merge(const h266_picture *src, const h266_picture *pre, const h266_sao_ctb_params *indep,
                             uint32_t pw, uint32_t ph, uint32_t bd, uint32_t log2, h266_sao_ctb_params *merged,
                             uint8_t *map) {
  const size_t chr = ((size_t)1 << log2) / 2;
  for (size_t i = 0; i < (size_t)pw * ph; ++i) merged[i] = indep[i];
  for (uint32_t ry = 0; ry < ph; ++ry)
    for (uint32_t rx = 0; rx < pw; ++rx) {
      const h266_sao_ctb_params in = merged[(size_t)ry * pw + rx];
      int64_t best = (int64_t)chroma_ctb_sse_with(src, pre, rx, ry, chr, bd, in.cb, in.cr) + 8 * sao_chroma_bits(in);
      uint8_t choice = 0;
      h266_sao_ctb bcb = in.cb, bcr = in.cr;
      if (rx > 0) {
        const h266_sao_ctb_params &l = merged[(size_t)ry * pw + rx - 1];
        const int64_t c = (int64_t)chroma_ctb_sse_with(src, pre, rx, ry, chr, bd, l.cb, l.cr) + 8 * 1;
        if (c < best) best = c, choice = 1, bcb = l.cb, bcr = l.cr;
      }
      if (ry > 0) {
        const h266_sao_ctb_params &u = merged[(size_t)(ry - 1) * pw + rx];
        const int64_t c = (int64_t)chroma_ctb_sse_with(src, pre, rx, ry, chr, bd, u.cb, u.cr) + 8 * 2;
        if (c < best) best = c, choice = 2, bcb = u.cb, bcr = u.cr;
      }
      map[(size_t)ry * pw + rx] = choice;
      merged[(size_t)ry * pw + rx].cb = bcb;
      merged[(size_t)ry * pw + rx].cr = bcr;
    }
}

// chroma_alf_decide_and_apply_clipped (src/alf_enc.rs:628-821) when cc is
// false, cc_alf_decide_and_apply_clipped (src/alf_enc.rs:935-1138) when true:
// per candidate (alt filter k, or CC filter k with idc k + 1) one apply_alf of
// the whole picture with that candidate on every CTB for component `comp`
// (1 = Cb, 2 = Cr), the CC trials on a copy whose luma is `pre_luma` (rec's
// luma layout); per CTB the lowest chroma SSE among {off, candidates} wins
// (strict <), its samples are copied into rec and `apply` records it.
static void chroma_decide(const h266_picture *src, h266_picture *rec, const uint16_t *pre_luma, h266_alf_ctb *apply,
                          const h266_alf_aps_data *aps, int comp, bool cc, uint32_t log2, uint32_t bd, uint32_t cfi,
                          const uint32_t *cols, size_t n_cols, const uint32_t *rows, size_t n_rows) {
  if (cfi == 0) return;
  size_t n_cand;
  if (!cc) {
    if (!aps->alf_chroma_filter_signal_flag) return;
    n_cand = aps->n_chroma_filters;
  } else {
    n_cand = comp == 1 ? aps->n_cc_cb_filters : aps->n_cc_cr_filters;
  }
  if (n_cand == 0) return;
  const uint32_t ctb = 1u << log2;
  const uint32_t wc = (rec->luma.width + ctb - 1) / ctb, hc = (rec->luma.height + ctb - 1) / ctb;
  const size_t n = (size_t)wc * hc;
  const uint32_t sw = cfi == 1 || cfi == 2 ? 2 : 1, sh = cfi == 1 ? 2 : 1;
  const size_t cw = ctb / sw, chh = ctb / sh;
  const h266_plane &sp = comp == 1 ? src->cb : src->cr;
  h266_plane &rp = comp == 1 ? rec->cb : rec->cr;
  std::vector<uint64_t> pre(n), per(n * n_cand);
  for (uint32_t ry = 0; ry < hc; ++ry)
    for (uint32_t rx = 0; rx < wc; ++rx)
      pre[(size_t)ry * wc + rx] = ctb_sse_y(sp, rp, (size_t)rx * ctb / sw, (size_t)ry * ctb / sh, cw, chh);
  h266_alf_aps_binding binding{};
  if (!cc) binding.chroma_aps = aps;
  else if (comp == 1) binding.cc_cb_aps = aps;
  else binding.cc_cr_aps = aps;
  h266_alf_config cfg{};
  cfg.alf_enabled = 1;
  cfg.cb_enabled = cfg.cc_cb_enabled = comp == 1;
  cfg.cr_enabled = cfg.cc_cr_enabled = comp == 2;
  cfg.bit_depth = bd;
  cfg.ctb_log2_size_y = log2;
  cfg.chroma_format_idc = cfi;
  const size_t nl = (size_t)rec->luma.stride * rec->luma.height, nb = (size_t)rec->cb.stride * rec->cb.height,
               nr = (size_t)rec->cr.stride * rec->cr.height;
  std::vector<std::vector<uint16_t>> kept(n_cand);
  std::vector<h266_alf_ctb> trial(n);
  for (size_t k = 0; k < n_cand; ++k) {
    std::vector<uint16_t> L(cc ? pre_luma : rec->luma.samples, (cc ? pre_luma : rec->luma.samples) + nl);
    std::vector<uint16_t> B(rec->cb.samples, rec->cb.samples + nb), Rr(rec->cr.samples, rec->cr.samples + nr);
    h266_picture t = *rec;
    t.luma.samples = L.data();
    t.cb.samples = B.data();
    t.cr.samples = Rr.data();
    for (size_t i = 0; i < n; ++i) {
      trial[i] = h266_alf_ctb{};
      if (!cc) {
        if (comp == 1) trial[i].cb_on = 1, trial[i].cb_alt_idx = (uint8_t)k;
        else trial[i].cr_on = 1, trial[i].cr_alt_idx = (uint8_t)k;
      } else {
        if (comp == 1) trial[i].cc_cb_idc = (uint8_t)(k + 1);
        else trial[i].cc_cr_idc = (uint8_t)(k + 1);
      }
    }
    h266_alf_picture ap{wc, hc, trial.data()};
    apply_alf_clipped(&t, &ap, &cfg, &binding, cols, n_cols, rows, n_rows);
    const h266_plane &tp = comp == 1 ? t.cb : t.cr;
    for (uint32_t ry = 0; ry < hc; ++ry)
      for (uint32_t rx = 0; rx < wc; ++rx)
        per[((size_t)ry * wc + rx) * n_cand + k] =
            ctb_sse_y(sp, tp, (size_t)rx * ctb / sw, (size_t)ry * ctb / sh, cw, chh);
    kept[k] = comp == 1 ? std::move(B) : std::move(Rr);
  }
  for (uint32_t ry = 0; ry < hc; ++ry)
    for (uint32_t rx = 0; rx < wc; ++rx) {
      const size_t idx = (size_t)ry * wc + rx;
      uint64_t best = pre[idx];
      int pick = -1;
      for (size_t k = 0; k < n_cand; ++k)
        if (per[idx * n_cand + k] < best) {
          best = per[idx * n_cand + k];
          pick = (int)k;
        }
      if (pick < 0) continue;
      const size_t x0 = (size_t)rx * ctb / sw, y0 = (size_t)ry * ctb / sh;
      const size_t w = std::min<size_t>(cw, rp.width > x0 ? rp.width - x0 : 0);
      const size_t h = std::min<size_t>(chh, rp.height > y0 ? rp.height - y0 : 0);
      for (size_t y = 0; y < h; ++y)
        std::memcpy(rp.samples + (y0 + y) * rp.stride + x0, kept[pick].data() + (y0 + y) * rp.stride + x0, w * 2);
      h266_alf_ctb &e = apply[idx];
      if (!cc) {
        if (comp == 1) e.cb_on = 1, e.cb_alt_idx = (uint8_t)pick;
        else e.cr_on = 1, e.cr_alt_idx = (uint8_t)pick;
      } else {
        if (comp == 1) e.cc_cb_idc = (uint8_t)(pick + 1);
        else e.cc_cr_idc = (uint8_t)(pick + 1);
      }
    }
}

}  // namespace oracle

// ---------------------------------------------------------------------------
// C API for the tests (ctypes).  Host memory only.
// ---------------------------------------------------------------------------
extern "C" {

int oracle_beta_prime(int q) { return oracle::beta_prime(q); }
int oracle_tc_prime(int q) { return oracle::tc_prime(q); }
int oracle_scale_tc(int tcp, uint32_t bd) { return oracle::scale_tc(tcp, bd); }
int oracle_scale_beta(int bp, uint32_t bd) { return oracle::scale_beta(bp, bd); }
int oracle_resolve_clip_value(uint32_t bd, uint32_t idx) { return oracle::resolve_clip_value(bd, (uint8_t)idx); }
void oracle_table_45(int y, int ctb, int apply, int *out) { oracle::table_45(y, ctb, apply != 0, out); }
void oracle_table_46(int y, int h, int apply, int *out) { oracle::table_46(y, h, apply != 0, out); }
void oracle_cc_alf_table_47(int y, int ctb, int apply, int *out) { oracle::cc_alf_table_47(y, ctb, apply != 0, out); }
void oracle_transpose_idx_table(int t, int *out) {
  const int *p = oracle::transpose_idx_table(t);
  for (int k = 0; k < 12; ++k) out[k] = p[k];
}
// fixed_filter_coeff_row, src/alf_fixed.rs:173-185; returns 0 for None.
int oracle_fixed_filter_coeff_row(uint32_t set, uint32_t cls, int *out) {
  if (set >= 16 || cls >= 25) return 0;
  const signed char *r = oracle::kAlfFixFiltCoeff[oracle::kAlfClassToFiltMap[set][cls]];
  for (int k = 0; k < 12; ++k) out[k] = r[k];
  return 1;
}
int oracle_class_to_filt_map(uint32_t set, uint32_t cls) { return oracle::kAlfClassToFiltMap[set][cls]; }
void oracle_derive_luma_classification(const uint16_t *pre, uint64_t stride, int ph, const int *clip, uint32_t rx,
                                       uint32_t ry, uint32_t ctb, uint32_t bd, uint8_t *filt, uint8_t *tr) {
  oracle::derive_luma_classification(pre, (size_t)stride, ph, clip, rx, ry, ctb, bd, filt, tr);
}

int oracle_derive_lmcs(const h266_lmcs_data *d, uint32_t bd, h266_lmcs_derived *o) { return oracle::derive_lmcs(d, bd, o); }
uint32_t oracle_lmcs_idx_y_inv(const h266_lmcs_derived *l, uint32_t s, uint32_t mn, uint32_t mx) {
  return oracle::idx_y_inv(l, s, mn, mx);
}
uint32_t oracle_lmcs_inverse_map(const h266_lmcs_derived *l, uint32_t s, uint32_t idx) { return oracle::inverse_map(l, s, idx); }
int64_t oracle_lmcs_forward_map(const h266_lmcs_derived *l, uint32_t s) { return oracle::forward_map(l, s); }
uint32_t oracle_lmcs_scale_chroma_residual(const h266_lmcs_derived *l, int64_t pred, int64_t res, uint32_t vs) {
  return oracle::scale_chroma_residual(l, pred, res, vs);
}
void oracle_lmcs_inverse_map_luma(h266_picture *pic, const h266_lmcs_derived *l, uint32_t mn, uint32_t mx) {
  oracle::lmcs_inverse_plane(pic->luma, l, mn, mx);
}

void oracle_apply_deblocking_clipped(h266_picture *pic, const h266_deblock_cu *cus, uint64_t n,
                                     const h266_deblock_cu *ccus, uint64_t nc, const h266_deblock_mv_grid *mv,
                                     const h266_deblock_params *params, uint32_t cfi, const uint32_t *cols,
                                     uint64_t n_cols, const uint32_t *rows, uint64_t n_rows) {
  oracle::apply_deblocking_clipped(pic, cus, n, ccus, nc, mv, params, cfi, cols, n_cols, rows, n_rows, nullptr, true);
}

// Edge segments in the reference's processing order (one record = 14 int32):
// c_idx, vertical, qx, qy, bS, mfl_p, mfl_q, beta, tc, ctb_row, plt_p, plt_q, cu_idx, off.
// Writes at most `cap` records and returns the total count.
uint64_t oracle_deblock_edge_log(const h266_picture *pic, const h266_deblock_cu *cus, uint64_t n,
                                 const h266_deblock_cu *ccus, uint64_t nc, const h266_deblock_mv_grid *mv,
                                 const h266_deblock_params *params, uint32_t cfi, const uint32_t *cols,
                                 uint64_t n_cols, const uint32_t *rows, uint64_t n_rows, int32_t *out, uint64_t cap) {
  std::vector<oracle::EdgeRec> log;
  h266_picture tmp = *pic;
  oracle::apply_deblocking_clipped(&tmp, cus, n, ccus, nc, mv, params, cfi, cols, n_cols, rows, n_rows, &log, false);
  for (uint64_t i = 0; i < log.size() && i < cap; ++i) std::memcpy(out + 14 * i, &log[i], 14 * sizeof(int32_t));
  return log.size();
}

// Re-apply logged edge segments in a caller-given order (test of the ordering
// argument the GPU deblocker relies on).  Vertical segments must come before
// horizontal ones of the same plane in `order`.
void oracle_deblock_replay(h266_picture *pic, const int32_t *recs, const uint64_t *order, uint64_t n) {
  for (uint64_t t = 0; t < n; ++t) {
    const int32_t *r = recs + 14 * order[t];
    h266_plane &hp = r[0] == 0 ? pic->luma : (r[0] == 1 ? pic->cb : pic->cr);
    oracle::Plane pl = oracle::mk(hp);
    bool vert = r[1] != 0;
    if (r[0] == 0)
      oracle::run_luma_filter(pl, r[2], r[3], r[7], r[8], (uint32_t)r[5], (uint32_t)r[6], vert, r[9] != 0, r[10] != 0,
                              r[11] != 0);
    else
      oracle::run_chroma_filter(pl, r[2], r[3], r[7], r[8], r[4], (uint32_t)r[5], (uint32_t)r[6], vert, r[10] != 0,
                                r[11] != 0);
  }
}

void oracle_apply_sao_clipped(h266_picture *pic, const h266_sao_picture *sp, const h266_sao_config *cfg,
                              const uint32_t *col_bd, uint64_t n_col, const uint32_t *row_bd, uint64_t n_row) {
  oracle::apply_sao_clipped(pic, sp, cfg, col_bd, n_col, row_bd, n_row);
}

void oracle_apply_alf_clipped(h266_picture *pic, const h266_alf_picture *ap, const h266_alf_config *cfg,
                              const h266_alf_aps_binding *b, const uint32_t *col_bd, uint64_t n_col,
                              const uint32_t *row_bd, uint64_t n_row) {
  oracle::apply_alf_clipped(pic, ap, cfg, b, col_bd, n_col, row_bd, n_row);
}

void oracle_apply_in_loop_filters(h266_picture *pic, const h266_in_loop_filter_args *a) { oracle::chain(pic, a); }

int oracle_lmcs_forward_map_rects(h266_picture *pic, const h266_lmcs_derived *l, const h266_rect *rects, uint64_t n) {
  return oracle::lmcs_forward_map_rects(pic->luma, l, rects, n) ? 0 : -1;
}
void oracle_lmcs_chroma_var_scale(const h266_picture *pic, const h266_lmcs_derived *l, uint32_t mn, uint32_t mx,
                                  uint32_t ctb_size_y, const h266_lmcs_cvs_block *b, uint64_t n, uint32_t *out) {
  const uint32_t size_y = std::min<uint32_t>(ctb_size_y, 64);
  for (uint64_t i = 0; i < n; ++i) out[i] = oracle::lmcs_chroma_var_scale(pic->luma, l, mn, mx, size_y, b[i]);
}
void oracle_lmcs_add_chroma_residual(h266_picture *pic, uint32_t bd, const int32_t *res,
                                     const h266_chroma_res_block *b, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i) oracle::add_chroma_residual(pic, bd, res, b[i]);
}
uint64_t oracle_output_convert(const h266_picture *pic, const h266_crop_window *c, uint32_t cfi, uint32_t bd,
                               uint8_t *out) {
  return oracle::output_convert(pic, *c, cfi, bd, out);
}

int oracle_sao_eo_category(int r, int n0, int n1) { return oracle::eo_category(r, n0, n1); }

void oracle_sao_decide_picture(const h266_picture *src, const h266_picture *rec, uint32_t log2, uint32_t bd,
                               int luma_on, int chroma_on, h266_sao_ctb_params *out) {
  oracle::sao_decide_picture(src, rec, log2, bd, luma_on != 0, chroma_on != 0, out);
}

void oracle_sao_chroma_merge(const h266_picture *src, const h266_picture *pre, const h266_sao_ctb_params *indep,
                             uint32_t pw, uint32_t ph, uint32_t bd, uint32_t log2, h266_sao_ctb_params *merged,
                             uint8_t *map) {
  oracle::sao_chroma_merge(src, pre, indep, pw, ph, bd, log2, merged, map);
}

void oracle_chroma_alf_decide(const h266_picture *src, h266_picture *rec, const uint16_t *pre_luma,
                              h266_alf_ctb *apply, const h266_alf_aps_data *aps, int comp, int cc, uint32_t log2,
                              uint32_t bd, uint32_t cfi, const uint32_t *cols, uint64_t n_cols, const uint32_t *rows,
                              uint64_t n_rows) {
  oracle::chroma_decide(src, rec, pre_luma, apply, aps, comp, cc != 0, log2, bd, cfi, cols, n_cols, rows, n_rows);
}

void oracle_alf_decide_and_apply(const h266_picture *src, h266_picture *rec, const h266_alf_aps_data *aps,
                                 uint32_t log2, uint32_t bd, uint32_t cfi, const uint32_t *cols, uint64_t n_cols,
                                 const uint32_t *rows, uint64_t n_rows, h266_alf_ctb *decisions, uint64_t *sse) {
  oracle::alf_decide_and_apply(src, rec, aps, log2, bd, cfi, cols, n_cols, rows, n_rows, decisions, sse);
}

// CPU baseline: n pictures spread over `threads` std::threads (one picture per
// task).  Returns the thread count used.
int oracle_apply_in_loop_filters_mt(uint32_t n, h266_picture *const *pics, const h266_in_loop_filter_args *const *args,
                                    int threads) {
  if (threads < 1) threads = 1;
  std::vector<std::thread> ts;
  std::atomic<uint32_t> next{0};
  for (int t = 0; t < threads; ++t)
    ts.emplace_back([&]() {
      for (;;) {
        uint32_t i = next.fetch_add(1);
        if (i >= n) break;
        oracle::chain(pics[i], args[i]);
      }
    });
  for (auto &t : ts) t.join();
  return threads;
}

}  // extern "C"
