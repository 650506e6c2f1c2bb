// SAO + ALF + CC-ALF tile pass, packed-arithmetic form (the default for
// BitDepth <= 14, |coefficients| <= 127 and 4:2:0 / 4:0:0 chroma; other inputs
// use the scalar pass in sao_alf.cu).
//
// Same semantics as the scalar pass (reads deblocked planes, writes final
// planes; post-SAO samples clamped into the CTB's ALF fetch rectangle), with a
// different organisation aimed at integer issue rate:
//  * tiles of TW x 32 luma samples (TW = 64 when the CTB allows it);
//  * SAO parameters of the 3x3 CTB neighbourhood cached in shared memory;
//  * ALF classification from per-2x2-cell Laplacian sums shared by the four
//    blocks whose windows contain the cell; only the two block rows next to
//    the CTB's virtual boundary (their windows and padding differ, src/alf.rs:
//    864-901) are summed directly;
//  * the 7x7 and 5x5 diamonds work on pairs of horizontally adjacent samples
//    packed in one 32-bit register: per tap the clipped differences of both
//    pixels are formed with two 16x2 add-max / add-min operations, the two
//    symmetric taps added as 16x2, and the coefficient applied per pixel with
//    dp2a; coefficients, clip values and their negations are pre-permuted per
//    (class, transposeIdx) on the host and held in registers per 4x4 block.
#include <initializer_list>

#include "internal.h"

namespace h266 {
namespace {

constexpr int TH = 32;
constexpr int NT = 256;

__device__ __forceinline__ int clampd(int v, int lo, int hi) { return min(max(v, lo), hi); }
__device__ __forceinline__ int sgn(int v) { return (v > 0) - (v < 0); }

// One component's SAO parameters of one CTB in the form the per-sample step
// needs: band offsets; for edge offset the offset per 2 + sign + sign (the
// edgeIdx remap of eq. 154 folded in), the shared-memory offset of the first
// neighbour (the second is its negation), and the rectangle of samples whose
// two neighbours lie inside the picture and the clip rectangle.
struct SaoLocal {
  int type, band, bd_shift;
  int off[4];   // band offset per band index 0..3 after the band position
  int eo[5];    // edge offset per 2 + sign(c - a) + sign(c - b)
  int nb;       // smem offset of the first neighbour (row pitch of the component's window)
  int ex0, ey0, ex1, ey1;  // [ex0, ex1) x [ey0, ey1): both neighbours available
};

template <int W>
struct Smem {
  static constexpr int DLW = W + 16, DLH = TH + 8;  // deblocked luma [X0-8, X1+8) x [Y0-4, Y1+4)
  static constexpr int SLW = W + 8, SLH = TH + 6;   // post-SAO luma [X0-4, X1+4) x [Y0-3, Y1+3)
  static constexpr int CW = W / 2 + 2, CH = TH / 2 + 2;  // 2x2 Laplacian cells
  static constexpr int DCW = W / 2 + 16, DCH = TH / 2 + 6;  // deblocked chroma [x-8, x+8) x [y-3, y+3)
  static constexpr int SCW = W / 2 + 8, SCH = TH / 2 + 4;   // post-SAO chroma [x-4, x+4) x [y-2, y+2)
  alignas(16) uint16_t dL[DLH * DLW];
  alignas(16) uint16_t sL[SLH * SLW];
  alignas(16) uint4 cell[CH * CW];  // sh, sv, sd0, sd1 over the cell's two checkerboard positions
  alignas(16) uint16_t dC[2][DCH * DCW];
  alignas(16) uint16_t sC[2][SCH * SCW];
  uint8_t cls_f[(TH / 4) * (W / 4)], cls_t[(TH / 4) * (W / 4)];
  SaoLocal sao[3][9];
};

// Fills one SaoLocal from the CTB's SAO parameters (src/sao.rs:504-626):
// hPos / vPos of eq. 152 per class, and the clip rectangle `rect` (component
// samples) intersected with the picture.
__device__ __forceinline__ void sao_local(SaoLocal &s, const SaoCtbDev &p, int pitch, int rx0, int ry0, int rx1,
                                          int ry1, int bd) {
  s.type = p.type;
  s.band = p.band_pos;
  s.bd_shift = bd - 5;
  for (int k = 0; k < 4; ++k) s.off[k] = p.off[k];
  // edgeIdx = 2 + sign + sign, remapped 0 -> 1, 1 -> 2, 2 -> 0 (eq. 154); offset edgeIdx - 1
  s.eo[0] = p.off[0];
  s.eo[1] = p.off[1];
  s.eo[2] = 0;
  s.eo[3] = p.off[2];
  s.eo[4] = p.off[3];
  const int h0 = p.eo_class == 0 ? -1 : (p.eo_class == 1 ? 0 : (p.eo_class == 2 ? -1 : 1));
  const int v0 = p.eo_class == 0 ? 0 : -1;
  s.nb = v0 * pitch + h0;
  const int ah = h0 < 0 ? -h0 : h0, av = v0 < 0 ? -v0 : v0;
  s.ex0 = rx0 + ah;
  s.ex1 = rx1 - ah;
  s.ey0 = ry0 + av;
  s.ey1 = ry1 - av;
}

// §8.8.4.2 for one sample at (x, y) whose pre-SAO value is *d (shared memory).
__device__ __forceinline__ int sao_one(const SaoLocal &p, int x, int y, int maxv, const uint16_t *d) {
  const int c = *d;
  if (p.type == 1) {
    const int k = ((c >> p.bd_shift) - p.band) & 31;
    return clampd(k < 4 ? c + p.off[k] : c, 0, maxv);
  }
  if (x < p.ex0 || x >= p.ex1 || y < p.ey0 || y >= p.ey1) return clampd(c, 0, maxv);
  return clampd(c + p.eo[2 + sgn(c - d[p.nb]) + sgn(c - d[-p.nb])], 0, maxv);
}

// Copies the HH x WW window at (x0, y0) of plane P (coordinates clamped into
// the plane) to dst with row pitch WW; whole 16-byte vectors when the window's
// columns lie inside the plane and the plane is aligned.
template <int WW, int HH>
__device__ __forceinline__ void load_window(uint16_t *dst, const DPlane &P, int x0, int y0) {
  static_assert(WW % 8 == 0, "whole vectors per row");
  const bool vec = x0 >= 0 && x0 + WW <= P.w && (x0 & 7) == 0 && ((uintptr_t)P.s & 15) == 0 && (P.stride & 7) == 0;
  if (vec) {
    constexpr int NV = WW / 8;
    for (int i = threadIdx.x; i < HH * NV; i += NT) {
      const int r = i / NV, c = (i - r * NV) * 8;
      const int gy = clampd(y0 + r, 0, P.h - 1);
      *reinterpret_cast<uint4 *>(dst + r * WW + c) = *reinterpret_cast<const uint4 *>(P.s + (int64_t)gy * P.stride + x0 + c);
    }
  } else {
    for (int i = threadIdx.x; i < HH * WW; i += NT) {
      const int r = i / WW, c = i - r * WW;
      const int gx = clampd(x0 + c, 0, P.w - 1), gy = clampd(y0 + r, 0, P.h - 1);
      dst[i] = P.s[(int64_t)gy * P.stride + gx];
    }
  }
}

// Pair of samples (col, col + 1) of a shared-memory row; DC fixes the parity
// of col (col = even base + DC).
template <int DC>
__device__ __forceinline__ uint32_t pair_at(const uint16_t *row, int even_base) {
  const int col = even_base + DC;
  if constexpr ((DC & 1) == 0) {
    return *reinterpret_cast<const uint32_t *>(row + col);
  } else {
    const uint32_t a = *reinterpret_cast<const uint32_t *>(row + col - 1);
    const uint32_t b = *reinterpret_cast<const uint32_t *>(row + col + 1);
    return __byte_perm(a, b, 0x5432);
  }
}

// clip(n - cur, -c, c) for both 16-bit lanes
__device__ __forceinline__ uint32_t clipd(uint32_t n, uint32_t ncur, uint32_t c2, uint32_t nc2) {
  return __viaddmin_s16x2(__viaddmax_s16x2(n, ncur, nc2), 0u, c2);
}
__device__ __forceinline__ uint32_t add2(uint32_t a, uint32_t b) { return __viaddmax_s16x2(a, b, 0x80008000u); }
__device__ __forceinline__ uint32_t neg2(uint32_t a) { return __viaddmax_s16x2(~a, 0x00010001u, 0x80008000u); }

template <int DX>
__device__ __forceinline__ void luma_tap(const uint16_t *up, const uint16_t *dn, int c0, const uint32_t ncur[2],
                                         uint32_t c2, uint32_t nc2, uint32_t f, int acc[4]) {
  // tap at (DX, +dy) on row `up`, mirrored tap at (-DX, -dy) on row `dn`
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const uint32_t a = clipd(pair_at<DX>(up, c0 + 2 * q), ncur[q], c2, nc2);
    const uint32_t b = clipd(pair_at<-DX>(dn, c0 + 2 * q), ncur[q], c2, nc2);
    const uint32_t s = add2(a, b);
    acc[2 * q] = __dp2a_lo((int)s, (int)f, acc[2 * q]);
    acc[2 * q + 1] = __dp2a_lo((int)s, (int)(f << 8), acc[2 * q + 1]);
  }
}

template <int DX>
__device__ __forceinline__ void chroma_tap(const uint16_t *up, const uint16_t *dn, int c0, uint32_t ncur, uint32_t c2,
                                           uint32_t nc2, uint32_t f, int acc[2]) {
  const uint32_t a = clipd(pair_at<DX>(up, c0), ncur, c2, nc2);
  const uint32_t b = clipd(pair_at<-DX>(dn, c0), ncur, c2, nc2);
  const uint32_t s = add2(a, b);
  acc[0] = __dp2a_lo((int)s, (int)f, acc[0]);
  acc[1] = __dp2a_lo((int)s, (int)(f << 8), acc[1]);
}

constexpr uint64_t pack4(std::initializer_list<int> v) {
  uint64_t r = 0;
  int i = 0;
  for (int x : v) r |= (uint64_t)x << (4 * i++);
  return r;
}
constexpr uint32_t pack2(std::initializer_list<int> v) {
  uint32_t r = 0;
  int i = 0;
  for (int x : v) r |= (uint32_t)x << (2 * i++);
  return r;
}

// Class of one block from its four direction sums (eqs. 1463-1482, src/alf.rs:954-1007).
__device__ __forceinline__ void classify(int sh, int sv, int sd0, int sd1, int ac, int bd, uint8_t &f_out,
                                         uint8_t &t_out) {
  int hv1, hv0, dhv, d1, d0, dd;
  if (sv > sh) { hv1 = sv; hv0 = sh; dhv = 1; } else { hv1 = sh; hv0 = sv; dhv = 3; }
  if (sd0 > sd1) { d1 = sd0; d0 = sd1; dd = 0; } else { d1 = sd1; d0 = sd0; dd = 2; }
  const bool pd = (long long)d1 * hv0 > (long long)hv1 * d0;
  const int hvd1 = pd ? d1 : hv1, hvd0 = pd ? d0 : hv0;
  const int dir1 = pd ? dd : dhv, dir2 = pd ? dhv : dd;
  const int dir_s = hvd1 * 2 > 9 * hvd0 ? 2 : (hvd1 > 2 * hvd0 ? 1 : 0);
  const long long act = ((long long)(sh + sv) * ac) >> (bd - 1);
  const int avg = (int)(act > 15 ? 15 : act);
  // varTab (eq. 1480) packed 4 bits per entry, transposeTable 2 bits per entry
  constexpr uint64_t kVarTab = pack4({0, 1, 2, 2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3, 4});
  constexpr uint32_t kTransposeTable = pack2({0, 1, 0, 2, 2, 3, 1, 3});
  int f = (int)((kVarTab >> (avg * 4)) & 0xF);
  if (dir_s != 0) f += (((dir1 & 1) << 1) + dir_s) * 5;
  f_out = (uint8_t)f;
  t_out = (uint8_t)((kTransposeTable >> ((dir1 * 2 + (dir2 >> 1)) * 2)) & 3);
}

// Chroma ALF (5x5 diamond, Table 46) and CC-ALF (Table 47) of one pair of
// chroma samples (tile column i2, i2 + 1, tile row jj) of plane `comp`.
template <int W>
__device__ __forceinline__ void chroma_pair(const Pass2Args &a, const Smem<W> &sm, int comp, int i2, int jj, int cf,
                                            int ccf, int xc0, int yc0, int y_ctb, int ctb, int ph, int bd, int maxv) {
  using S = Smem<W>;
  const DPlane CD = a.dst[comp];
  const int ctb_c = ctb / 2, y_ctb_c = y_ctb / 2;
  const int gy = yc0 + jj, gx = xc0 + i2;
  const int r = jj + 2, c0 = i2 + 4;
  const uint16_t *R0 = &sm.sC[comp - 1][r * S::SCW];
  const uint32_t cur = pair_at<0>(R0, c0);
  int v[2] = {(int)(cur & 0xFFFF), (int)(cur >> 16)};
  if (cf >= 0) {
    const int jr = gy - y_ctb_c;
    int s2 = 7, y1 = 1, y2 = 2;  // Table 46 (line-buffer arms always applied)
    if (jr == ctb_c - 2 || jr == ctb_c - 3) { s2 = 10; y1 = y2 = 0; }
    else if (jr == ctb_c - 1 || jr == ctb_c - 4) { y2 = 1; }
    const uint32_t *ct = a.tables.chroma_packed + max(cf, 0) * 18;
    const uint32_t ncur = neg2(cur);
    int acc[2] = {0, 0};
    const uint16_t *U1 = R0 - y1 * S::SCW, *D1 = R0 + y1 * S::SCW, *U2 = R0 - y2 * S::SCW, *D2 = R0 + y2 * S::SCW;
    chroma_tap<0>(D2, U2, c0, ncur, ct[0], ct[1], ct[2], acc);
    chroma_tap<1>(D1, U1, c0, ncur, ct[3], ct[4], ct[5], acc);
    chroma_tap<0>(D1, U1, c0, ncur, ct[6], ct[7], ct[8], acc);
    chroma_tap<-1>(D1, U1, c0, ncur, ct[9], ct[10], ct[11], acc);
    chroma_tap<2>(R0, R0, c0, ncur, ct[12], ct[13], ct[14], acc);
    chroma_tap<1>(R0, R0, c0, ncur, ct[15], ct[16], ct[17], acc);
    const int round = 1 << (s2 - 1);
    v[0] = clampd(v[0] + ((acc[0] + round) >> s2), 0, maxv);
    v[1] = clampd(v[1] + ((acc[1] + round) >> s2), 0, maxv);
  }
  if (ccf >= 0) {  // CC-ALF from post-SAO luma (Table 47, src/alf.rs:447-523)
    const int *cc = a.tables.cc_coeff[comp - 1][max(ccf, 0)];
    const int half = 1 << (bd - 1);
    const int yline = (gy - y_ctb_c) * 2;
    const bool lbb = !(gy * 2 + ctb >= ph && (ph - y_ctb) <= ctb - 4);
    int yp1 = 1, yp2 = 2;
    if (lbb) {
      if (yline == ctb - 5 || yline == ctb - 4) { yp1 = 0; yp2 = 0; }
      else if (yline == ctb - 6 || yline == ctb - 3) { yp2 = 1; }
    }
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const uint16_t *L = &sm.sL[(2 * jj + 3) * S::SLW + 2 * (i2 + p) + 4];
      const int ctr = L[0];
      int sum = cc[0] * ((int)L[-yp1 * S::SLW] - ctr);
      sum += cc[1] * ((int)L[-1] - ctr);
      sum += cc[2] * ((int)L[1] - ctr);
      sum += cc[3] * ((int)L[yp1 * S::SLW - 1] - ctr);
      sum += cc[4] * ((int)L[yp1 * S::SLW] - ctr);
      sum += cc[5] * ((int)L[yp1 * S::SLW + 1] - ctr);
      sum += cc[6] * ((int)L[yp2 * S::SLW] - ctr);
      v[p] = clampd(v[p] + clampd((sum + 64) >> 7, -half, half - 1), 0, maxv);
    }
  }
  if (gy < CD.h) {
    uint16_t *out = CD.s + (int64_t)gy * CD.stride + gx;
    if (gx < CD.w) out[0] = (uint16_t)v[0];
    if (gx + 1 < CD.w) out[1] = (uint16_t)v[1];
  }
}

// One tile (index `tile` of the picture's tile grid) of the pass.  Phases,
// each ended by one barrier: (1) SAO parameters and every plane's deblocked
// window; (2) post-SAO windows of all planes; (3) luma Laplacian cells and
// the chroma planes' ALF / CC-ALF (their inputs are complete after 2);
// (4) luma classes; (5) the 7x7 luma filter.
// Laplacian sums per 2x2 cell of the luma window `sm.sL` (unpadded rows).
template <class S>
__device__ __forceinline__ void luma_cells(S &sm) {
  for (int i = threadIdx.x; i < S::CH * S::CW; i += NT) {
    const int cy = i / S::CW, cx = i - cy * S::CW;
    uint4 g = make_uint4(0, 0, 0, 0);
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      const int r = 2 * cy + d + 1;  // sL row of the position: y = Y0 - 2 + 2cy + d
      const int c = 2 * cx + d + 2;  // sL col: x = X0 - 2 + 2cx + d
      const uint16_t *row = &sm.sL[r * S::SLW + c];
      const int c2 = 2 * row[0];
      g.x += abs(c2 - row[-1] - row[1]);
      g.y += abs(c2 - row[-S::SLW] - row[S::SLW]);
      g.z += abs(c2 - row[-S::SLW - 1] - row[S::SLW + 1]);
      g.w += abs(c2 - row[-S::SLW + 1] - row[S::SLW - 1]);
    }
    sm.cell[i] = g;
  }
}

// Class and transposeIdx of every 4x4 block of the tile (src/alf.rs:750-1008).
template <int W, class S>
__device__ __forceinline__ void luma_classes(S &sm, int Y0, int y_ctb, int ctb, int ph, int bd) {
  const bool bottom = y_ctb + ctb >= ph;
  const bool carve = !bottom || (ph - y_ctb) > ctb - 4;
  const int vb = y_ctb + ctb - 4;
  constexpr int NB = (TH / 4) * (W / 4);
  for (int b = threadIdx.x; b < NB; b += NT) {
    const int bx = b % (W / 4), by = b / (W / 4);
    const int y4 = Y0 + 4 * by - y_ctb;
    if (y4 == ctb - 8 || y4 == ctb - 4) {  // virtual-boundary rows: windows and padding differ
      int min_y = -2, max_y = 5, ac = 2;
      if (y4 == ctb - 8 && carve) { max_y = 3; ac = 3; }
      else if (y4 == ctb - 4 && carve) { min_y = 0; ac = 3; }
      const bool top_pad = y4 == ctb - 4, bot_pad = y4 == ctb - 8;
      auto pad = [&](int gy) {
        if (top_pad) gy = max(gy, vb);
        if (bot_pad) gy = min(gy, vb - 1);
        return gy - (Y0 - 3);
      };
      int sh = 0, sv = 0, sd0 = 0, sd1 = 0;
      for (int j = min_y; j <= max_y; ++j) {
        const int gy = y_ctb + y4 + j;
        const uint16_t *rc = &sm.sL[pad(gy) * S::SLW], *ru = &sm.sL[pad(gy - 1) * S::SLW],
                       *rd = &sm.sL[pad(gy + 1) * S::SLW];
        for (int i = (j & 1) ? -1 : -2; i <= 5; i += 2) {
          const int c = 4 * bx + i + 4;
          const int c2 = 2 * rc[c];
          sh += abs(c2 - rc[c - 1] - rc[c + 1]);
          sv += abs(c2 - ru[c] - rd[c]);
          sd0 += abs(c2 - ru[c - 1] - rd[c + 1]);
          sd1 += abs(c2 - ru[c + 1] - rd[c - 1]);
        }
      }
      classify(sh, sv, sd0, sd1, ac, bd, sm.cls_f[b], sm.cls_t[b]);
    } else {
      uint4 s = make_uint4(0, 0, 0, 0);
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const uint4 g = sm.cell[(2 * by + r) * S::CW + 2 * bx + c];
          s.x += g.x;
          s.y += g.y;
          s.z += g.z;
          s.w += g.w;
        }
      classify((int)s.x, (int)s.y, (int)s.z, (int)s.w, 2, bd, sm.cls_f[b], sm.cls_t[b]);
    }
  }
}

// The 7x7 diamond on one run of 4 samples (tile row j, block column bx) with
// one block's packed taps; `yr` is the row inside its CTB.  out[] receives the
// filtered samples (src/alf.rs:652-743, Table 45 arms always applied).
template <class S>
__device__ __forceinline__ void luma_run(const S &sm, int j, int bx, int yr, int ctb, const uint32_t c2[12],
                                         const uint32_t nc2[12], const uint32_t f[12], int maxv, int out[4]) {
  int shift = 7, y1 = 1, y2 = 2, y3 = 3;
  if (yr == ctb - 5 || yr == ctb - 4) { shift = 10; y1 = y2 = y3 = 0; }
  else if (yr == ctb - 6 || yr == ctb - 3) { y2 = y3 = 1; }
  else if (yr == ctb - 7 || yr == ctb - 2) { y3 = 2; }
  const int r = j + 3;
  const int c0 = 4 * bx + 4;
  const uint16_t *R0 = &sm.sL[r * S::SLW];
  const uint16_t *U1 = R0 - y1 * S::SLW, *D1 = R0 + y1 * S::SLW;
  const uint16_t *U2 = R0 - y2 * S::SLW, *D2 = R0 + y2 * S::SLW;
  const uint16_t *U3 = R0 - y3 * S::SLW, *D3 = R0 + y3 * S::SLW;
  const uint32_t cur[2] = {pair_at<0>(R0, c0), pair_at<0>(R0, c0 + 2)};
  const uint32_t ncur[2] = {neg2(cur[0]), neg2(cur[1])};
  int acc[4] = {0, 0, 0, 0};
  luma_tap<0>(D3, U3, c0, ncur, c2[0], nc2[0], f[0], acc);
  luma_tap<1>(D2, U2, c0, ncur, c2[1], nc2[1], f[1], acc);
  luma_tap<0>(D2, U2, c0, ncur, c2[2], nc2[2], f[2], acc);
  luma_tap<-1>(D2, U2, c0, ncur, c2[3], nc2[3], f[3], acc);
  luma_tap<2>(D1, U1, c0, ncur, c2[4], nc2[4], f[4], acc);
  luma_tap<1>(D1, U1, c0, ncur, c2[5], nc2[5], f[5], acc);
  luma_tap<0>(D1, U1, c0, ncur, c2[6], nc2[6], f[6], acc);
  luma_tap<-1>(D1, U1, c0, ncur, c2[7], nc2[7], f[7], acc);
  luma_tap<-2>(D1, U1, c0, ncur, c2[8], nc2[8], f[8], acc);
  luma_tap<3>(R0, R0, c0, ncur, c2[9], nc2[9], f[9], acc);
  luma_tap<2>(R0, R0, c0, ncur, c2[10], nc2[10], f[10], acc);
  luma_tap<1>(R0, R0, c0, ncur, c2[11], nc2[11], f[11], acc);
  const int round = 1 << (shift - 1);
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int cv = (int)((cur[p >> 1] >> ((p & 1) * 16)) & 0xFFFF);
    out[p] = clampd(cv + ((acc[p] + round) >> shift), 0, maxv);
  }
}

// The 12 symmetric tap sums (n+ - cur) + (n- - cur) of one 4-sample run,
// packed per pixel pair, without clipping: the form every filter set whose
// clip values never bind shares (clipIdx 0 gives 2^BitDepth, above any
// |n - cur| of in-range samples).  Same taps and Table 45 rows as luma_run.
template <class S>
__device__ __forceinline__ void luma_sums(const S &sm, int j, int bx, int yr, int ctb, uint32_t sum[2][12],
                                          uint32_t cur[2], int &shift) {
  int y1 = 1, y2 = 2, y3 = 3;
  shift = 7;
  if (yr == ctb - 5 || yr == ctb - 4) { shift = 10; y1 = y2 = y3 = 0; }
  else if (yr == ctb - 6 || yr == ctb - 3) { y2 = y3 = 1; }
  else if (yr == ctb - 7 || yr == ctb - 2) { y3 = 2; }
  const int c0 = 4 * bx + 4;
  const uint16_t *R0 = &sm.sL[(j + 3) * S::SLW];
  const uint16_t *U1 = R0 - y1 * S::SLW, *D1 = R0 + y1 * S::SLW;
  const uint16_t *U2 = R0 - y2 * S::SLW, *D2 = R0 + y2 * S::SLW;
  const uint16_t *U3 = R0 - y3 * S::SLW, *D3 = R0 + y3 * S::SLW;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int c = c0 + 2 * q;
    cur[q] = pair_at<0>(R0, c);
    const uint32_t nc = neg2(cur[q]);
    auto tap = [&](uint32_t up, uint32_t dn) {
      return add2(__viaddmax_s16x2(up, nc, 0x80008000u), __viaddmax_s16x2(dn, nc, 0x80008000u));
    };
    sum[q][0] = tap(pair_at<0>(D3, c), pair_at<0>(U3, c));
    sum[q][1] = tap(pair_at<1>(D2, c), pair_at<-1>(U2, c));
    sum[q][2] = tap(pair_at<0>(D2, c), pair_at<0>(U2, c));
    sum[q][3] = tap(pair_at<-1>(D2, c), pair_at<1>(U2, c));
    sum[q][4] = tap(pair_at<2>(D1, c), pair_at<-2>(U1, c));
    sum[q][5] = tap(pair_at<1>(D1, c), pair_at<-1>(U1, c));
    sum[q][6] = tap(pair_at<0>(D1, c), pair_at<0>(U1, c));
    sum[q][7] = tap(pair_at<-1>(D1, c), pair_at<1>(U1, c));
    sum[q][8] = tap(pair_at<-2>(D1, c), pair_at<2>(U1, c));
    sum[q][9] = tap(pair_at<3>(R0, c), pair_at<-3>(R0, c));
    sum[q][10] = tap(pair_at<2>(R0, c), pair_at<-2>(R0, c));
    sum[q][11] = tap(pair_at<1>(R0, c), pair_at<-1>(R0, c));
  }
}

template <int W, bool DO_SAO, bool DO_ALF>
__device__ __forceinline__ void sao_alf_tile(const Pass2Args &a, int tile) {
  using S = Smem<W>;
  extern __shared__ __align__(16) uint8_t smem_raw[];
  S &sm = *reinterpret_cast<S *>(smem_raw);
  const int tid = threadIdx.x;
  const int tx = tile % a.tiles_x, ty = tile / a.tiles_x;
  const int X0 = tx * W, Y0 = ty * TH;
  const int bd = a.bit_depth, maxv = (1 << bd) - 1;
  const int log2 = a.ctb_log2, ctb = 1 << log2;
  const int rx = X0 >> log2, ry = Y0 >> log2;
  const int y_ctb = ry << log2;
  const int pw = a.pic_w, ph = a.pic_h;
  const bool in_grid = rx < a.w_ctbs && ry < a.h_ctbs;
  const CtbDev *me = in_grid ? &a.ctbs[ry * a.w_ctbs + rx] : nullptr;
  int rect[4] = {0, 0, pw, ph};
  if (me) {
    rect[0] = me->rect[0];
    rect[1] = me->rect[1];
    rect[2] = me->rect[2];
    rect[3] = me->rect[3];
  }
  const int rx0 = max(rect[0], 0), ry0 = max(rect[1], 0), rx1 = min(rect[2], pw), ry1 = min(rect[3], ph);
  constexpr int TWC = W / 2, THC = TH / 2;
  const int xc0 = X0 / 2, yc0 = Y0 / 2;
  bool chroma_on[2] = {false, false};  // the tile has chroma samples of that plane
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const DPlane &CS = a.src[c + 1];
    chroma_on[c] = a.chroma && CS.w > 0 && CS.h > 0 && xc0 < CS.w && yc0 < CS.h;
  }

  // ---- (1) SAO parameters of the 3x3 CTB neighbourhood; deblocked windows
  if (tid < 27) {
    const int comp = tid / 9, n = tid % 9;
    const int nx = rx + n % 3 - 1, ny = ry + n / 3 - 1;
    SaoLocal &s = sm.sao[comp][n];
    s.type = 0;
    const bool used = comp == 0 ? a.sao_luma : a.sao_chroma;
    if (DO_SAO && used && nx >= 0 && ny >= 0 && nx < a.w_ctbs && ny < a.h_ctbs) {
      const CtbDev &c = a.ctbs[ny * a.w_ctbs + nx];
      const int sw = comp ? 2 : 1;
      const int cw = comp ? a.src[comp].w : a.src[0].w, ch = comp ? a.src[comp].h : a.src[0].h;
      int q0 = 0, q1 = 0, q2 = cw, q3 = ch;  // clip rectangle in component samples, within the picture
      if (a.has_clip) {
        q0 = max(q0, c.rect[0] / sw);
        q1 = max(q1, c.rect[1] / sw);
        q2 = min(q2, (c.rect[2] + sw - 1) / sw);
        q3 = min(q3, (c.rect[3] + sw - 1) / sw);
      }
      sao_local(s, c.sao[comp], comp ? S::DCW : S::DLW, q0, q1, q2, q3, bd);
    }
  }
  const DPlane LS = a.src[0], LD = a.dst[0];
  load_window<S::DLW, S::DLH>(sm.dL, LS, X0 - 8, Y0 - 4);
#pragma unroll
  for (int c = 0; c < 2; ++c)
    if (chroma_on[c]) load_window<S::DCW, S::DCH>(sm.dC[c], a.src[c + 1], xc0 - 8, yc0 - 3);
  __syncthreads();
  int any_sao[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    int any = 0;
    for (int n = 0; n < 9; ++n) any |= sm.sao[c][n].type;
    any_sao[c] = any;
  }

  // ---- (2) post-SAO windows, clamped into the fetch rectangle
  for (int i = tid; i < S::SLH * S::SLW; i += NT) {
    const int r = i / S::SLW, c = i - r * S::SLW;
    const int ax = clampd(X0 - 4 + c, rx0, rx1 - 1), ay = clampd(Y0 - 3 + r, ry0, ry1 - 1);
    const uint16_t *d = &sm.dL[(ay - (Y0 - 4)) * S::DLW + ax - (X0 - 8)];
    int v = *d;
    if (any_sao[0]) {
      const SaoLocal &p = sm.sao[0][((ay >> log2) - ry + 1) * 3 + ((ax >> log2) - rx + 1)];
      if (p.type) v = sao_one(p, ax, ay, maxv, d);
    }
    sm.sL[i] = (uint16_t)v;
  }
  const int crx0 = rect[0] / 2, cry0 = rect[1] / 2, crx1 = (rect[2] + 1) / 2, cry1 = (rect[3] + 1) / 2;
#pragma unroll
  for (int cc = 0; cc < 2; ++cc) {
    if (!chroma_on[cc]) continue;
    const DPlane &CS = a.src[cc + 1];
    const int cx0 = max(crx0, 0), cy0 = max(cry0, 0), cx1 = min(crx1, CS.w), cy1 = min(cry1, CS.h);
    for (int i = tid; i < S::SCH * S::SCW; i += NT) {
      const int r = i / S::SCW, c = i - r * S::SCW;
      const int ax = clampd(xc0 - 4 + c, cx0, cx1 - 1), ay = clampd(yc0 - 2 + r, cy0, cy1 - 1);
      const uint16_t *d = &sm.dC[cc][(ay - (yc0 - 3)) * S::DCW + ax - (xc0 - 8)];
      int v = *d;
      if (any_sao[cc + 1]) {
        const SaoLocal &p = sm.sao[cc + 1][(((ay * 2) >> log2) - ry + 1) * 3 + (((ax * 2) >> log2) - rx + 1)];
        if (p.type) v = sao_one(p, ax, ay, maxv, d);
      }
      sm.sC[cc][i] = (uint16_t)v;
    }
  }
  __syncthreads();

  // ---- (3) luma Laplacian sums per 2x2 cell (unpadded rows); chroma ALF / CC-ALF
  const bool luma_alf = DO_ALF && me && me->luma_set >= 0;
  if (luma_alf) luma_cells(sm);
  {
    // both chroma planes, one pair of samples per (plane, pair) item
    constexpr int PAIRS = (TWC / 2) * THC;  // per plane
    for (int it = tid; it < 2 * PAIRS; it += NT) {
      const int cc = it / PAIRS, q = it - cc * PAIRS;
      if (!chroma_on[cc]) continue;
      const int cf = (DO_ALF && me) ? me->chroma_filt[cc] : -1;
      const int ccf = (DO_ALF && me) ? me->cc_filt[cc] : -1;
      chroma_pair<W>(a, sm, cc + 1, (q % (TWC / 2)) * 2, q / (TWC / 2), cf, ccf, xc0, yc0, y_ctb, ctb, ph, bd, maxv);
    }
  }
  if (!luma_alf) {
    for (int p = tid; p < TH * W; p += NT) {
      const int i = p % W, j = p / W;
      const int gx = X0 + i, gy = Y0 + j;
      if (gx < LD.w && gy < LD.h) LD.s[(int64_t)gy * LD.stride + gx] = sm.sL[(j + 3) * S::SLW + i + 4];
    }
    return;
  }
  __syncthreads();

  // ---- (4) classes
  luma_classes<W>(sm, Y0, y_ctb, ctb, ph, bd);
  __syncthreads();

  // ---- (5) 7x7 diamond, 4-pixel runs; every thread keeps one block's taps
  constexpr int RUNS = TH * W / 4;
  constexpr int RPT = RUNS / NT;  // runs per thread: 1 (W = 32) or 2 (W = 64)
  constexpr int TPB = 4 / RPT;    // threads per 4x4 block
  const int b = tid / TPB;
  const int bx = b % (W / 4), by = b / (W / 4);
  const uint32_t *tab = a.tables.luma_packed + ((size_t)me->luma_set * 100 + sm.cls_f[b] * 4 + sm.cls_t[b]) * 36;
  uint32_t c2[12], nc2[12], f[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    c2[k] = __ldg(tab + 3 * k);
    nc2[k] = __ldg(tab + 3 * k + 1);
    f[k] = __ldg(tab + 3 * k + 2);
  }
#pragma unroll
  for (int rr = 0; rr < RPT; ++rr) {
    const int jr = (tid % TPB) * RPT + rr;  // row inside the block
    const int j = 4 * by + jr;               // tile row
    const int gy = Y0 + j;
    if (gy < LD.h) {
      int o[4];
      luma_run(sm, j, bx, gy - y_ctb, ctb, c2, nc2, f, maxv, o);
      uint16_t *out = LD.s + (int64_t)gy * LD.stride + X0 + 4 * bx;
#pragma unroll
      for (int p = 0; p < 4; ++p)
        if (X0 + 4 * bx + p < LD.w) out[p] = (uint16_t)o[p];
    }
  }
}

template <int W, bool DO_SAO, bool DO_ALF>
__global__ void __launch_bounds__(NT, 4) k_sao_alf_packed(const __grid_constant__ Pass2Args a) {
  sao_alf_tile<W, DO_SAO, DO_ALF>(a, blockIdx.x);
}

// Many pictures in one grid: CTAs [first[i], first[i + 1]) are the tiles of
// picture i, whose parameters are args[i].
template <int W, bool DO_SAO, bool DO_ALF>
__global__ void __launch_bounds__(NT, 4) k_sao_alf_packed_batch(const Pass2Args *__restrict__ args,
                                                             const uint32_t *__restrict__ first, int n) {
  __shared__ Pass2Args s_args;  // the picture's parameters, read once per CTA
  int lo = 0, hi = n;            // first[lo] <= blockIdx.x < first[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (first[mid] <= blockIdx.x) lo = mid;
    else hi = mid;
  }
  static_assert(sizeof(Pass2Args) % 4 == 0, "word copy");
  const uint32_t *src = reinterpret_cast<const uint32_t *>(args + lo);
  uint32_t *dst = reinterpret_cast<uint32_t *>(&s_args);
  for (int i = threadIdx.x; i < (int)(sizeof(Pass2Args) / 4); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  sao_alf_tile<W, DO_SAO, DO_ALF>(s_args, (int)(blockIdx.x - first[lo]));
}

// ---- encoder luma ALF trials (src/alf_enc.rs:185-528)
//
// The reference runs one full apply_alf per candidate filter set (16 fixed
// sets, plus the APS set) on a copy of the picture and sums SSE_Y per CTB
// against the original.  Luma ALF output depends only on the pre-ALF samples
// and the CTB's own filter set, so one tile pass serves every trial: it
// stages the pre-ALF window once, classifies the 4x4 blocks once, then
// filters the tile with each trial's taps and adds the squared errors of its
// samples into per-(CTB, trial) sums; nothing is written back.  Column 0 of a
// CTB's row is the pre-ALF SSE (the "off" option).
template <int W>
struct TrialSmem {
  static constexpr int SLW = W + 8, SLH = TH + 6;        // pre-ALF luma [X0-4, X1+4) x [Y0-3, Y1+3)
  static constexpr int CW = W / 2 + 2, CH = TH / 2 + 2;  // 2x2 Laplacian cells
  alignas(16) uint16_t sL[SLH * SLW];
  alignas(16) uint4 cell[CH * CW];
  uint8_t cls_f[(TH / 4) * (W / 4)], cls_t[(TH / 4) * (W / 4)];
  alignas(8) unsigned long long sse[kAlfMaxTrials + 1];
};

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <int W>
__global__ void __launch_bounds__(NT, 2) k_alf_luma_trials(const __grid_constant__ Pass2Args a, const DPlane orig,
                                                           int trials, int cols, unsigned long long *__restrict__ sse) {
  using S = TrialSmem<W>;
  __shared__ S sm;
  const int tid = threadIdx.x, tile = blockIdx.x;
  const int tx = tile % a.tiles_x, ty = tile / a.tiles_x;
  const int X0 = tx * W, Y0 = ty * TH;
  const int bd = a.bit_depth, maxv = (1 << bd) - 1;
  const int log2 = a.ctb_log2, ctb = 1 << log2;
  const int rx = X0 >> log2, ry = Y0 >> log2;
  if (rx >= a.w_ctbs || ry >= a.h_ctbs) return;  // uniform per CTA
  const int y_ctb = ry << log2;
  const int pw = a.pic_w, ph = a.pic_h;
  const CtbDev &me = a.ctbs[ry * a.w_ctbs + rx];
  const int rx0 = max((int)me.rect[0], 0), ry0 = max((int)me.rect[1], 0);
  const int rx1 = min((int)me.rect[2], pw), ry1 = min((int)me.rect[3], ph);
  const DPlane LS = a.src[0];
  int wide = 0;  // a sample above 2^BitDepth - 1 (outside the picture format): clips may bind for every set
  for (int i = tid; i < S::SLH * S::SLW; i += NT) {  // clamped into the fetch rectangle (sample(), src/alf.rs:1093-1110)
    const int r = i / S::SLW, c = i - r * S::SLW;
    const int ax = clampd(X0 - 4 + c, rx0, rx1 - 1), ay = clampd(Y0 - 3 + r, ry0, ry1 - 1);
    const uint16_t v = LS.s[(int64_t)ay * LS.stride + ax];
    wide |= v > maxv;
    sm.sL[i] = v;
  }
  if (tid <= trials) sm.sse[tid] = 0;
  wide = __syncthreads_or(wide);
  luma_cells(sm);
  __syncthreads();
  luma_classes<W>(sm, Y0, y_ctb, ctb, ph, bd);
  __syncthreads();

  constexpr int RUNS = TH * W / 4;
  constexpr int RPT = RUNS / NT;
  constexpr int TPB = 4 / RPT;
  const int b = tid / TPB;
  const int bx = b % (W / 4), by = b / (W / 4);
  // the SSE window is the CTB inside both planes (ctb_sse_y, src/alf_enc.rs:79-105)
  const int vw = min(orig.w, pw), vh = min(orig.h, ph);
  int org[RPT][4];
  unsigned long long e0 = 0;
#pragma unroll
  for (int rr = 0; rr < RPT; ++rr) {
    const int j = 4 * by + (tid % TPB) * RPT + rr, gy = Y0 + j;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const int gx = X0 + 4 * bx + p;
      const bool in = gx < vw && gy < vh;
      org[rr][p] = in ? (int)orig.s[(int64_t)gy * orig.stride + gx] : -1;
      if (in) {
        const int d = org[rr][p] - (int)sm.sL[(j + 3) * S::SLW + 4 * bx + p + 4];
        e0 += (unsigned long long)((long long)d * d);
      }
    }
  }
  e0 = warp_sum(e0);
  if ((tid & 31) == 0) atomicAdd(&sm.sse[0], e0);
  const int cls = sm.cls_f[b] * 4 + sm.cls_t[b];
  int first = 0;  // first trial of the clipped path
  if (!wide) {
    // fixed sets 0..15 (clipIdx 0): tap sums once, then 12 dp2a per pixel pair per set
    first = min(trials, 16);
    uint32_t sum[RPT][2][12], cur[RPT][2];
    int shift[RPT];
#pragma unroll
    for (int rr = 0; rr < RPT; ++rr) {
      const int j = 4 * by + (tid % TPB) * RPT + rr;
      luma_sums(sm, j, bx, Y0 + j - y_ctb, ctb, sum[rr], cur[rr], shift[rr]);
    }
    const uint32_t *tab0 = a.tables.luma_packed + (size_t)cls * 36 + 2;  // coefficient words of trial t at + t * 3600
    uint32_t fn[12];  // the next trial's coefficients, loaded while the current trial runs
#pragma unroll
    for (int k = 0; k < 12; ++k) fn[k] = first > 0 ? __ldg(tab0 + 3 * k) : 0u;
    for (int t = 0; t < first; ++t) {
      uint32_t f[12];
#pragma unroll
      for (int k = 0; k < 12; ++k) f[k] = fn[k];
      if (t + 1 < first) {
#pragma unroll
        for (int k = 0; k < 12; ++k) fn[k] = __ldg(tab0 + (size_t)(t + 1) * 3600 + 3 * k);
      }
      unsigned long long e = 0;
#pragma unroll
      for (int rr = 0; rr < RPT; ++rr) {
        const int round = 1 << (shift[rr] - 1);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          int lo = 0, hi = 0;
#pragma unroll
          for (int k = 0; k < 12; ++k) {
            lo = __dp2a_lo((int)sum[rr][q][k], (int)f[k], lo);
            hi = __dp2a_lo((int)sum[rr][q][k], (int)(f[k] << 8), hi);
          }
          const int v0 = clampd((int)(cur[rr][q] & 0xFFFF) + ((lo + round) >> shift[rr]), 0, maxv);
          const int v1 = clampd((int)(cur[rr][q] >> 16) + ((hi + round) >> shift[rr]), 0, maxv);
          if (org[rr][2 * q] >= 0) {
            const int d = org[rr][2 * q] - v0;
            e += (unsigned long long)((long long)d * d);
          }
          if (org[rr][2 * q + 1] >= 0) {
            const int d = org[rr][2 * q + 1] - v1;
            e += (unsigned long long)((long long)d * d);
          }
        }
      }
      e = warp_sum(e);
      if ((tid & 31) == 0) atomicAdd(&sm.sse[1 + t], e);
    }
  }
  for (int t = first; t < trials; ++t) {
    const uint32_t *tab = a.tables.luma_packed + ((size_t)t * 100 + cls) * 36;
    uint32_t c2[12], nc2[12], f[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      c2[k] = __ldg(tab + 3 * k);
      nc2[k] = __ldg(tab + 3 * k + 1);
      f[k] = __ldg(tab + 3 * k + 2);
    }
    unsigned long long e = 0;
#pragma unroll
    for (int rr = 0; rr < RPT; ++rr) {
      const int j = 4 * by + (tid % TPB) * RPT + rr;
      int o[4];
      luma_run(sm, j, bx, Y0 + j - y_ctb, ctb, c2, nc2, f, maxv, o);
#pragma unroll
      for (int p = 0; p < 4; ++p)
        if (org[rr][p] >= 0) {
          const int d = org[rr][p] - o[p];
          e += (unsigned long long)((long long)d * d);
        }
    }
    e = warp_sum(e);
    if ((tid & 31) == 0) atomicAdd(&sm.sse[1 + t], e);
  }
  __syncthreads();
  if (tid <= trials) atomicAdd(&sse[(size_t)(ry * a.w_ctbs + rx) * cols + tid], sm.sse[tid]);
}

// Per CTB the lowest SSE among {off, trial 0, ...} (strict <: earlier options
// win ties, src/alf_enc.rs:276-292, 482-498); the commit pass then filters
// the chosen CTBs with their sets.  Trials not run (an APS without luma
// filters leaves the samples as they are) take the pre-ALF SSE.
__global__ void k_alf_luma_decide(CtbDev *__restrict__ ctbs, int n, unsigned long long *__restrict__ sse, int cols,
                                  int trials_run, int16_t *__restrict__ decision) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long *row = sse + (size_t)i * cols;
  for (int t = trials_run; t < cols - 1; ++t) row[1 + t] = row[0];
  unsigned long long best = row[0];
  int pick = -1;
  for (int t = 0; t < cols - 1; ++t)
    if (row[1 + t] < best) {
      best = row[1 + t];
      pick = t;
    }
  ctbs[i].luma_set = (int16_t)pick;
  decision[i] = (int16_t)pick;
}

template <int W>
int launch_w(cudaStream_t st, const Pass2Args &in, bool do_sao, bool do_alf) {
  static_assert(sizeof(Smem<W>) <= 48 * 1024, "fits the default dynamic shared-memory limit");
  Pass2Args a = in;
  a.tiles_x = (a.ext_w + W - 1) / W;
  a.tiles_y = (a.ext_h + TH - 1) / TH;
  const unsigned n = (unsigned)(a.tiles_x * a.tiles_y);
  const size_t shm = sizeof(Smem<W>);
  auto go = [&](auto kern) -> int {
    kern<<<n, NT, shm, st>>>(a);
    H266_CUDA(cudaGetLastError());
    return H266_OK;
  };
  if (do_sao && do_alf) return go(k_sao_alf_packed<W, true, true>);
  if (do_sao) return go(k_sao_alf_packed<W, true, false>);
  if (do_alf) return go(k_sao_alf_packed<W, false, true>);
  return go(k_sao_alf_packed<W, false, false>);
}

}  // namespace

int pass2_packed_variant(Pass2Args &a, bool do_sao, bool do_alf, uint32_t *ctas) {
  const int W = a.ctb_log2 >= 6 ? 64 : 32;
  a.tiles_x = (a.ext_w + W - 1) / W;
  a.tiles_y = (a.ext_h + TH - 1) / TH;
  *ctas = a.ext_w > 0 && a.ext_h > 0 ? (uint32_t)(a.tiles_x * a.tiles_y) : 0;
  return (W == 64 ? 4 : 0) + (do_sao ? 2 : 0) + (do_alf ? 1 : 0);
}

int launch_pass2_packed_batch(cudaStream_t st, int variant, const Pass2Args *d_args, const uint32_t *d_first, int n,
                              uint32_t ctas, uint64_t *launches) {
  if (!ctas || n <= 0) return H266_OK;
  auto go = [&](auto kern, size_t shm) -> int {
    kern<<<ctas, NT, shm, st>>>(d_args, d_first, n);
    H266_CUDA(cudaGetLastError());
    ++*launches;
    return H266_OK;
  };
  switch (variant) {
    case 7: return go(k_sao_alf_packed_batch<64, true, true>, sizeof(Smem<64>));
    case 6: return go(k_sao_alf_packed_batch<64, true, false>, sizeof(Smem<64>));
    case 5: return go(k_sao_alf_packed_batch<64, false, true>, sizeof(Smem<64>));
    case 4: return go(k_sao_alf_packed_batch<64, false, false>, sizeof(Smem<64>));
    case 3: return go(k_sao_alf_packed_batch<32, true, true>, sizeof(Smem<32>));
    case 2: return go(k_sao_alf_packed_batch<32, true, false>, sizeof(Smem<32>));
    case 1: return go(k_sao_alf_packed_batch<32, false, true>, sizeof(Smem<32>));
    default: return go(k_sao_alf_packed_batch<32, false, false>, sizeof(Smem<32>));
  }
}

int launch_alf_luma_trials(cudaStream_t st, const Pass2Args &in, const DPlane &orig, int trials, int cols,
                           unsigned long long *d_sse, uint64_t *launches) {
  if (in.ext_w <= 0 || in.ext_h <= 0) return H266_OK;
  if (trials < 0 || trials > kAlfMaxTrials || cols < trials + 1)
    return set_error(H266_ERR_INVALID_ARGUMENT, "ALF trials: bad trial count");
  Pass2Args a = in;
  const int W = a.ctb_log2 >= 6 ? 64 : 32;
  a.tiles_x = (a.ext_w + W - 1) / W;
  a.tiles_y = (a.ext_h + TH - 1) / TH;
  const unsigned n = (unsigned)(a.tiles_x * a.tiles_y);
  if (W == 64) k_alf_luma_trials<64><<<n, NT, 0, st>>>(a, orig, trials, cols, d_sse);
  else k_alf_luma_trials<32><<<n, NT, 0, st>>>(a, orig, trials, cols, d_sse);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

int launch_alf_luma_decide(cudaStream_t st, CtbDev *d_ctbs, int n, unsigned long long *d_sse, int cols, int trials_run,
                           int16_t *d_decision, uint64_t *launches) {
  if (n <= 0) return H266_OK;
  k_alf_luma_decide<<<(n + 127) / 128, 128, 0, st>>>(d_ctbs, n, d_sse, cols, trials_run, d_decision);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

int launch_pass2_packed(cudaStream_t st, const Pass2Args &a, bool do_sao, bool do_alf, uint64_t *launches) {
  if (a.ext_w <= 0 || a.ext_h <= 0) return H266_OK;
  const int rc = a.ctb_log2 >= 6 ? launch_w<64>(st, a, do_sao, do_alf) : launch_w<32>(st, a, do_sao, do_alf);
  if (rc == H266_OK) ++*launches;
  return rc;
}

}  // namespace h266
