// Device helpers shared by the chain's SAO / ALF / CC-ALF tile kernel
// (sao_alf3.cu) and the encoder's luma ALF trial kernel (sao_alf2.cu).
//
// Packed coefficient words (AlfTablesDev::luma_packed / chroma_packed): per
// tap three words -- the clip value in both 16-bit lanes, its negation in both
// lanes, and the coefficient as a signed byte in bytes 0 and 3, so that
// __dp2a_lo(s, f) weights the low lane of a packed pair of tap sums and
// __dp2a_hi(s, f) the high lane.
#pragma once

#include <initializer_list>

#include "internal.h"

namespace h266 {
namespace tile {

__device__ __forceinline__ int clampd(int v, int lo, int hi) { return min(max(v, lo), hi); }
__device__ __forceinline__ int sgn(int v) { return (v > 0) - (v < 0); }

// One component's SAO parameters of one CTB in the form the per-sample step
// needs: band offsets; for edge offset the offset per 2 + sign + sign (the
// edgeIdx remap of eq. 154 folded in), the shared-memory offset of the first
// neighbour (the second is its negation), and the rectangle of samples whose
// two neighbours lie inside the picture and the clip rectangle.  tlo / thi
// hold the same offsets as a signed-byte table (bytes 0..3 of tlo, then thi)
// indexed by the band index 0..3 (4 = no offset) or by 4 + sign + sign.
struct SaoLocal {
  int type, band, bd_shift;
  int off[4];   // band offset per band index 0..3 after the band position
  int eo[5];    // edge offset per 2 + sign(c - a) + sign(c - b)
  int nb;       // smem offset of the first neighbour (row pitch of the component's window)
  int ex0, ey0, ex1, ey1;  // [ex0, ex1) x [ey0, ey1): both neighbours available
  uint32_t tlo, thi;
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
  auto b = [](int v) { return (uint32_t)(v & 0xFF); };
  if (p.type == 1) {
    s.tlo = b(p.off[0]) | b(p.off[1]) << 8 | b(p.off[2]) << 16 | b(p.off[3]) << 24;
    s.thi = 0;
  } else {  // indexed by (sign + 2) + (sign + 2) = 2 + edgeIdx, so the table starts at byte 2
    s.tlo = b(s.eo[0]) << 16 | b(s.eo[1]) << 24;
    s.thi = b(s.eo[2]) | b(s.eo[3]) << 8 | b(s.eo[4]) << 16;
  }
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
    acc[2 * q + 1] = __dp2a_hi((int)s, (int)f, acc[2 * q + 1]);
  }
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

// Laplacian sums per 2x2 cell of the luma window `sL` (unpadded rows):
// cell (cx, cy) covers positions (X0 - 2 + 2cx + d, Y0 - 2 + 2cy + d), d = 0, 1.
template <class S, int NT>
__device__ __forceinline__ void luma_cells(const uint16_t *sL, uint4 *cell) {
  for (int i = threadIdx.x; i < S::CH * S::CW; i += NT) {
    const int cy = i / S::CW, cx = i - cy * S::CW;
    uint4 g = make_uint4(0, 0, 0, 0);
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      const int r = 2 * cy + d + 1;  // sL row of the position: y = Y0 - 2 + 2cy + d
      const int c = 2 * cx + d + 2;  // sL col: x = X0 - 2 + 2cx + d
      const uint16_t *row = &sL[r * S::SLP + c];
      const int c2 = 2 * row[0];
      g.x += abs(c2 - row[-1] - row[1]);
      g.y += abs(c2 - row[-S::SLP] - row[S::SLP]);
      g.z += abs(c2 - row[-S::SLP - 1] - row[S::SLP + 1]);
      g.w += abs(c2 - row[-S::SLP + 1] - row[S::SLP - 1]);
    }
    cell[i] = g;
  }
}

// Class and transposeIdx of every 4x4 block of a W x TH tile (src/alf.rs:750-1008).
template <int W, int TH, class S, int NT>
__device__ __forceinline__ void luma_classes(const uint16_t *sL, const uint4 *cell, uint8_t *cls_f, uint8_t *cls_t,
                                             int Y0, int y_ctb, int ctb, int ph, int bd) {
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
        const uint16_t *rc = &sL[pad(gy) * S::SLP], *ru = &sL[pad(gy - 1) * S::SLP], *rd = &sL[pad(gy + 1) * S::SLP];
        for (int i = (j & 1) ? -1 : -2; i <= 5; i += 2) {
          const int c = 4 * bx + i + 4;
          const int c2 = 2 * rc[c];
          sh += abs(c2 - rc[c - 1] - rc[c + 1]);
          sv += abs(c2 - ru[c] - rd[c]);
          sd0 += abs(c2 - ru[c - 1] - rd[c + 1]);
          sd1 += abs(c2 - ru[c + 1] - rd[c - 1]);
        }
      }
      classify(sh, sv, sd0, sd1, ac, bd, cls_f[b], cls_t[b]);
    } else {
      uint4 s = make_uint4(0, 0, 0, 0);
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const uint4 g = cell[(2 * by + r) * S::CW + 2 * bx + c];
          s.x += g.x;
          s.y += g.y;
          s.z += g.z;
          s.w += g.w;
        }
      classify((int)s.x, (int)s.y, (int)s.z, (int)s.w, 2, bd, cls_f[b], cls_t[b]);
    }
  }
}

// Table 45 rows of a luma row `yr` inside its CTB (line-buffer arms always applied,
// src/alf.rs:694, 1117-1130): the filter shift and the row offsets y1..y3.
__device__ __forceinline__ void table45(int yr, int ctb, int &shift, int &y1, int &y2, int &y3) {
  shift = 7;
  y1 = 1;
  y2 = 2;
  y3 = 3;
  if (yr == ctb - 5 || yr == ctb - 4) { shift = 10; y1 = y2 = y3 = 0; }
  else if (yr == ctb - 6 || yr == ctb - 3) { y2 = y3 = 1; }
  else if (yr == ctb - 7 || yr == ctb - 2) { y3 = 2; }
}

// The 7x7 diamond on one run of 4 samples (window row j, block column bx) with
// one block's packed taps; `yr` is the row inside its CTB.  out[] receives the
// filtered samples (src/alf.rs:652-743, Table 45 arms always applied).
template <class S>
__device__ __forceinline__ void luma_run(const S &sm, int j, int bx, int yr, int ctb, const uint32_t c2[12],
                                         const uint32_t nc2[12], const uint32_t f[12], int maxv, int out[4]) {
  int shift, y1, y2, y3;
  table45(yr, ctb, shift, y1, y2, y3);
  const int r = j + 3;
  const int c0 = 4 * bx + 4;
  const uint16_t *R0 = &sm.sL[r * S::SLP];
  const uint16_t *U1 = R0 - y1 * S::SLP, *D1 = R0 + y1 * S::SLP;
  const uint16_t *U2 = R0 - y2 * S::SLP, *D2 = R0 + y2 * S::SLP;
  const uint16_t *U3 = R0 - y3 * S::SLP, *D3 = R0 + y3 * S::SLP;
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
  int y1, y2, y3;
  table45(yr, ctb, shift, y1, y2, y3);
  const int c0 = 4 * bx + 4;
  const uint16_t *R0 = &sm.sL[(j + 3) * S::SLP];
  const uint16_t *U1 = R0 - y1 * S::SLP, *D1 = R0 + y1 * S::SLP;
  const uint16_t *U2 = R0 - y2 * S::SLP, *D2 = R0 + y2 * S::SLP;
  const uint16_t *U3 = R0 - y3 * S::SLP, *D3 = R0 + y3 * S::SLP;
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

}  // namespace tile
}  // namespace h266
