// SAO (§8.8.4) and ALF (§8.8.5: 4x4 classification, 7x7 luma, 5x5 chroma,
// CC-ALF) as one tile pass.
//
// One CTA filters a 32x32 luma tile and its co-located chroma tiles.  Tiles
// never straddle a CTB (CTB sizes are 32, 64 or 128), so the CTB parameters,
// the ALF fetch-clip rectangle and the line-buffer virtual boundary are
// uniform over a tile.  The pass reads the deblocked planes (src) and writes
// the final planes (dst), which is the reference's snapshot semantics: SAO
// reads a pre-SAO copy (src/sao.rs:404-423), ALF and CC-ALF read a pre-ALF
// copy (src/alf.rs:265-276), so no sample of one tile depends on another
// tile's output.
//
// Shared-memory staging per tile:
//   dL  deblocked luma   [Y0-4, Y1+4) x [X0-4, X1+4)   (SAO needs +-1)
//   sL  post-SAO luma    [Y0-3, Y1+3) x [X0-3, X1+3)   (classification / 7x7 need +-3)
// Every sL cell holds the post-SAO value at its coordinates clamped into the
// tile's ALF fetch rectangle, which is exactly what the reference's clamped
// fetch `sample()` (src/alf.rs:1104-1109) returns; the filters then read sL
// without per-tap clamping.  Chroma uses the same scheme with +-3 / +-2.
#include "internal.h"

namespace h266 {
namespace {

constexpr int T = 32;           // luma tile edge
constexpr int DL = T + 8;       // dL edge
constexpr int SL = T + 6;       // sL edge
constexpr int DC = T + 6;       // dC edge (max, 4:4:4)
constexpr int SC = T + 4;       // sC edge (max)
constexpr int NTHREADS = 256;

__constant__ int8_t c_transpose[4][12] = {{0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11},
                                          {9, 4, 10, 8, 1, 5, 11, 7, 3, 0, 2, 6},
                                          {0, 3, 2, 1, 8, 7, 6, 5, 4, 9, 10, 11},
                                          {9, 8, 10, 4, 3, 7, 11, 5, 1, 0, 2, 6}};  // eqs. 1442-1445

__device__ __forceinline__ int clampd(int v, int lo, int hi) { return min(max(v, lo), hi); }
__device__ __forceinline__ int sgn(int v) { return (v > 0) - (v < 0); }

// §8.8.4.2 for one sample (apply_sao_ctb, src/sao.rs:504-626).  `at(dx, dy)`
// reads the pre-SAO plane around the sample; (x, y) are its plane coordinates,
// (pw, ph) the plane size and rect the sample's CTB clip rectangle.
template <class At>
__device__ __forceinline__ int sao_sample(const SaoCtbDev &p, int x, int y, int pw, int ph, const int rect[4],
                                          int bd, int maxv, At at) {
  const int c = at(0, 0);
  if (p.type == 1) {  // band offset, eq. 1434
    const int band = (c >> (bd - 5)) & 31;
    const int k = (band - p.band_pos) & 31;
    return k < 4 ? clampd(c + p.off[k], 0, maxv) : clampd(c, 0, maxv);
  }
  // edge offset, Table 44 + eqs. 1429-1432
  const int cls = p.eo_class & 3;
  const int h0 = cls == 0 ? -1 : (cls == 1 ? 0 : (cls == 2 ? -1 : 1));
  const int v0 = cls == 0 ? 0 : -1;
  const int h1 = -h0, v1 = -v0;
  const int nx0 = x + h0, ny0 = y + v0, nx1 = x + h1, ny1 = y + v1;
  const bool outside = nx0 < max(0, rect[0]) || nx1 < max(0, rect[0]) || ny0 < max(0, rect[1]) ||
                       ny1 < max(0, rect[1]) || nx0 >= min(pw, rect[2]) || nx1 >= min(pw, rect[2]) ||
                       ny0 >= min(ph, rect[3]) || ny1 >= min(ph, rect[3]);
  if (outside) return clampd(c, 0, maxv);
  int e = 2 + sgn(c - at(h0, v0)) + sgn(c - at(h1, v1));
  if (e <= 2) e = e == 2 ? 0 : e + 1;
  return e >= 1 ? clampd(c + p.off[e - 1], 0, maxv) : clampd(c, 0, maxv);
}

struct LumaCoef {
  int32_t coeff[25 * 12];
  int32_t clip[25 * 12];
};

template <bool DO_SAO, bool DO_ALF>
__global__ void __launch_bounds__(NTHREADS) k_sao_alf(const __grid_constant__ Pass2Args a) {
  __shared__ uint16_t dL[DL][DL + 2];
  __shared__ uint16_t sL[SL][SL + 2];
  __shared__ uint16_t dC[DC][DC + 2];
  __shared__ uint16_t sC[SC][SC + 2];
  __shared__ uint8_t cls_f[64], cls_t[64];
  __shared__ LumaCoef lc;

  const int tid = threadIdx.x;
  const int tx = blockIdx.x % a.tiles_x, ty = blockIdx.x / a.tiles_x;
  const int X0 = tx * T, Y0 = ty * T;
  const int bd = a.bit_depth, maxv = (1 << bd) - 1;
  const int log2 = a.ctb_log2, ctb = 1 << log2;
  const int rx = X0 >> log2, ry = Y0 >> log2;
  const bool in_grid = rx < a.w_ctbs && ry < a.h_ctbs;
  const CtbDev *me = in_grid ? &a.ctbs[ry * a.w_ctbs + rx] : nullptr;
  const int pw = a.pic_w, ph = a.pic_h;
  int rect[4] = {0, 0, pw, ph};
  if (me) {
    rect[0] = me->rect[0];
    rect[1] = me->rect[1];
    rect[2] = me->rect[2];
    rect[3] = me->rect[3];
  }
  const int x_ctb = rx << log2, y_ctb = ry << log2;

  // ------------------------------------------------------------ luma
  const DPlane LS = a.src[0], LD = a.dst[0];
  const bool have_luma = LS.w > 0 && LS.h > 0 && X0 < LS.w && Y0 < LS.h;  // tile starts inside the picture
  const bool luma_alf = DO_ALF && me && me->luma_set >= 0 && have_luma;
  const bool need_sl = have_luma;  // CC-ALF also reads sL
  if (need_sl) {
    for (int i = tid; i < DL * DL; i += NTHREADS) {
      const int r = i / DL, c = i % DL;
      const int gx = clampd(X0 - 4 + c, 0, LS.w - 1), gy = clampd(Y0 - 4 + r, 0, LS.h - 1);
      dL[r][c] = LS.s[(int64_t)gy * LS.stride + gx];
    }
    __syncthreads();
    for (int i = tid; i < SL * SL; i += NTHREADS) {
      const int r = i / SL, c = i % SL;
      // clamp into the fetch rectangle (and the picture)
      const int ax = clampd(X0 - 3 + c, max(rect[0], 0), min(rect[2], pw) - 1);
      const int ay = clampd(Y0 - 3 + r, max(rect[1], 0), min(rect[3], ph) - 1);
      const int lr = ay - (Y0 - 4), lcol = ax - (X0 - 4);
      int v = dL[lr][lcol];
      if (DO_SAO && a.sao_luma) {
        const int srx = ax >> log2, sry = ay >> log2;
        if (srx < a.w_ctbs && sry < a.h_ctbs) {
          const CtbDev &sc = a.ctbs[sry * a.w_ctbs + srx];
          if (sc.sao[0].type != 0) {
            const int big = 1 << 30;  // without tile bounds only the picture edge gates EO
            const int srect[4] = {a.has_clip ? (int)sc.rect[0] : 0, a.has_clip ? (int)sc.rect[1] : 0,
                                  a.has_clip ? (int)sc.rect[2] : big, a.has_clip ? (int)sc.rect[3] : big};
            v = sao_sample(sc.sao[0], ax, ay, LS.w, LS.h, srect, bd, maxv,
                           [&](int dx, int dy) { return (int)dL[lr + dy][lcol + dx]; });
          }
        }
      }
      sL[r][c] = (uint16_t)v;
    }
    __syncthreads();
  }

  if (have_luma && luma_alf) {
    // §8.8.5.3 classification (derive_luma_classification, src/alf.rs:822-1010):
    // 4 threads per 4x4 block, each summing two window rows.
    const bool bottom = y_ctb + ctb >= ph;
    const bool carve = !bottom || (ph - y_ctb) > ctb - 4;
    const int vb = y_ctb + ctb - 4;
    {
      const int b = tid >> 2, q = tid & 3;
      const int bx = b & 7, by = b >> 3;
      const int y4 = Y0 + 4 * by - y_ctb;  // CTB-relative
      int min_y = -2, max_y = 5, ac = 2;
      if (y4 == ctb - 8 && carve) {
        max_y = 3;
        ac = 3;
      } else if (y4 == ctb - 4 && carve) {
        min_y = 0;
        ac = 3;
      }
      const bool top_pad = y4 >= ctb - 4;
      const bool bot_pad = ctb - 4 - y4 > 0 && ctb - 4 - y4 < 5;
      auto pad = [&](int gy) {
        if (top_pad) gy = max(gy, vb);
        if (bot_pad) gy = min(gy, vb - 1);
        return gy - (Y0 - 3);
      };
      int sh = 0, sv = 0, sd0 = 0, sd1 = 0;
      for (int jj = q; jj < 8; jj += 4) {
        const int j = min_y + jj;
        if (j > max_y) break;
        const int gy = y_ctb + y4 + j;
        const int rc = pad(gy), ru = pad(gy - 1), rd = pad(gy + 1);
        for (int i = ((j & 1) ? -1 : -2); i <= 5; i += 2) {  // checkerboard: i and j of equal parity
          const int c = X0 + 4 * bx + i - (X0 - 3);
          const int c2 = 2 * sL[rc][c];
          sh += abs(c2 - sL[rc][c - 1] - sL[rc][c + 1]);
          sv += abs(c2 - sL[ru][c] - sL[rd][c]);
          sd0 += abs(c2 - sL[ru][c - 1] - sL[rd][c + 1]);
          sd1 += abs(c2 - sL[ru][c + 1] - sL[rd][c - 1]);
        }
      }
#pragma unroll
      for (int m = 1; m < 4; m <<= 1) {
        sh += __shfl_xor_sync(0xffffffffu, sh, m);
        sv += __shfl_xor_sync(0xffffffffu, sv, m);
        sd0 += __shfl_xor_sync(0xffffffffu, sd0, m);
        sd1 += __shfl_xor_sync(0xffffffffu, sd1, m);
      }
      if (q == 0) {
        int hv1, hv0, dhv, d1, d0, dd;
        if (sv > sh) { hv1 = sv; hv0 = sh; dhv = 1; } else { hv1 = sh; hv0 = sv; dhv = 3; }
        if (sd0 > sd1) { d1 = sd0; d0 = sd1; dd = 0; } else { d1 = sd1; d0 = sd0; dd = 2; }
        const bool pd = (long long)d1 * hv0 > (long long)hv1 * d0;
        const int hvd1 = pd ? d1 : hv1, hvd0 = pd ? d0 : hv0;
        const int dir1 = pd ? dd : dhv, dir2 = pd ? dhv : dd;
        const int dir_s = hvd1 * 2 > 9 * hvd0 ? 2 : (hvd1 > 2 * hvd0 ? 1 : 0);
        const long long act = ((long long)(sh + sv) * ac) >> (bd - 1);
        const int avg = (int)(act < 0 ? 0 : (act > 15 ? 15 : act));
        const int var_tab[16] = {0, 1, 2, 2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3, 4};
        const int tt[8] = {0, 1, 0, 2, 2, 3, 1, 3};
        int f = var_tab[avg];
        if (dir_s != 0) f += (((dir1 & 1) << 1) + dir_s) * 5;
        cls_f[b] = (uint8_t)f;
        cls_t[b] = (uint8_t)tt[dir1 * 2 + (dir2 >> 1)];
      }
    }
    for (int i = tid; i < 300; i += NTHREADS) {
      lc.coeff[i] = a.tables.luma_coeff[me->luma_set * 600 + i];
      lc.clip[i] = a.tables.luma_clip[me->luma_set * 600 + i];
    }
    __syncthreads();
    // §8.8.5.2 7x7 diamond (apply_alf_luma_ctb, src/alf.rs:652-724)
    for (int p = tid; p < T * T; p += NTHREADS) {
      const int i = p & (T - 1), j = p >> 5;
      const int gx = X0 + i, gy = Y0 + j;
      if (gx >= LD.w || gy >= LD.h) continue;
      const int jr = gy - y_ctb;
      int shift = 7, y1 = 1, y2 = 2, y3 = 3;  // Table 45, always with the line-buffer arms
      if (jr == ctb - 5 || jr == ctb - 4) { shift = 10; y1 = y2 = y3 = 0; }
      else if (jr == ctb - 6 || jr == ctb - 3) { y2 = y3 = 1; }
      else if (jr == ctb - 7 || jr == ctb - 2) { y3 = 2; }
      const int b = (j >> 2) * 8 + (i >> 2);
      const int f = cls_f[b];
      const int8_t *perm = c_transpose[cls_t[b]];
      const int32_t *co = &lc.coeff[f * 12];
      const int32_t *cl = &lc.clip[f * 12];
      const int r = j + 3, c = i + 3;
      const int cur = sL[r][c];
      auto tap = [&](int k, int dx, int dy) {
        const int lim = cl[perm[k]];
        return clampd((int)sL[r + dy][c + dx] - cur, -lim, lim) + clampd((int)sL[r - dy][c - dx] - cur, -lim, lim);
      };
      int sum = co[perm[0]] * tap(0, 0, y3);
      sum += co[perm[1]] * tap(1, 1, y2);
      sum += co[perm[2]] * tap(2, 0, y2);
      sum += co[perm[3]] * tap(3, -1, y2);
      sum += co[perm[4]] * tap(4, 2, y1);
      sum += co[perm[5]] * tap(5, 1, y1);
      sum += co[perm[6]] * tap(6, 0, y1);
      sum += co[perm[7]] * tap(7, -1, y1);
      sum += co[perm[8]] * tap(8, -2, y1);
      sum += co[perm[9]] * tap(9, 3, 0);
      sum += co[perm[10]] * tap(10, 2, 0);
      sum += co[perm[11]] * tap(11, 1, 0);
      const int v = cur + ((sum + (1 << (shift - 1))) >> shift);
      LD.s[(int64_t)gy * LD.stride + gx] = (uint16_t)clampd(v, 0, maxv);
    }
  } else if (have_luma) {
    for (int p = tid; p < T * T; p += NTHREADS) {
      const int i = p & (T - 1), j = p >> 5;
      const int gx = X0 + i, gy = Y0 + j;
      if (gx >= LD.w || gy >= LD.h) continue;
      // inside the picture the rect clamp is the identity for the tile's own samples
      LD.s[(int64_t)gy * LD.stride + gx] = sL[j + 3][i + 3];
    }
  }

  // ------------------------------------------------------------ chroma
  if (!a.chroma) return;
  const int sw = a.sub_w, shc = a.sub_h;
  const int twc = T / sw, thc = T / shc;
  const int xc0 = X0 / sw, yc0 = Y0 / shc;
  const int ctb_w_c = ctb / sw, ctb_h_c = ctb / shc;
  const int x_ctb_c = x_ctb / sw, y_ctb_c = y_ctb / shc;
  int crect[4] = {rect[0] / sw, rect[1] / shc, (rect[2] + sw - 1) / sw, (rect[3] + shc - 1) / shc};
  for (int comp = 1; comp <= 2; ++comp) {
    const DPlane CS = a.src[comp], CD = a.dst[comp];
    if (CS.w <= 0 || CS.h <= 0) continue;
    if (xc0 >= CS.w || yc0 >= CS.h) continue;
    const int cr0 = max(crect[0], 0), cr1 = max(crect[1], 0), cr2 = min(crect[2], CS.w), cr3 = min(crect[3], CS.h);
    __syncthreads();  // dC / sC reuse
    for (int i = tid; i < (thc + 6) * (twc + 6); i += NTHREADS) {
      const int r = i / (twc + 6), c = i % (twc + 6);
      const int gx = clampd(xc0 - 3 + c, 0, CS.w - 1), gy = clampd(yc0 - 3 + r, 0, CS.h - 1);
      dC[r][c] = CS.s[(int64_t)gy * CS.stride + gx];
    }
    __syncthreads();
    for (int i = tid; i < (thc + 4) * (twc + 4); i += NTHREADS) {
      const int r = i / (twc + 4), c = i % (twc + 4);
      const int ax = clampd(xc0 - 2 + c, cr0, cr2 - 1), ay = clampd(yc0 - 2 + r, cr1, cr3 - 1);
      const int lr = ay - (yc0 - 3), lcol = ax - (xc0 - 3);
      int v = dC[lr][lcol];
      if (DO_SAO && a.sao_chroma) {
        const int srx = (ax * sw) >> log2, sry = (ay * shc) >> log2;
        if (srx < a.w_ctbs && sry < a.h_ctbs) {
          const CtbDev &sc = a.ctbs[sry * a.w_ctbs + srx];
          if (sc.sao[comp].type != 0) {
            const int big = 1 << 30;
            const int srect[4] = {a.has_clip ? sc.rect[0] / sw : 0, a.has_clip ? sc.rect[1] / shc : 0,
                                  a.has_clip ? (sc.rect[2] + sw - 1) / sw : big,
                                  a.has_clip ? (sc.rect[3] + shc - 1) / shc : big};
            v = sao_sample(sc.sao[comp], ax, ay, CS.w, CS.h, srect, bd, maxv,
                           [&](int dx, int dy) { return (int)dC[lr + dy][lcol + dx]; });
          }
        }
      }
      sC[r][c] = (uint16_t)v;
    }
    __syncthreads();
    const int cf = (DO_ALF && me) ? me->chroma_filt[comp - 1] : -1;
    const int ccf = (DO_ALF && me && have_luma) ? me->cc_filt[comp - 1] : -1;
    const int *ccoef = cf >= 0 ? a.tables.chroma_coeff[cf] : nullptr;
    const int *cclip = cf >= 0 ? a.tables.chroma_clip[cf] : nullptr;
    const int *cc = ccf >= 0 ? a.tables.cc_coeff[comp - 1][ccf] : nullptr;
    const int half = 1 << (bd - 1);
    for (int p = tid; p < thc * twc; p += NTHREADS) {
      const int i = p % twc, j = p / twc;
      const int gx = xc0 + i, gy = yc0 + j;
      if (gx >= CD.w || gy >= CD.h) continue;
      const int r = j + 2, c = i + 2;
      const int cur = sC[r][c];
      int v = cur;
      if (cf >= 0) {  // §8.8.5.4 5x5 diamond (apply_alf_chroma_ctb, src/alf.rs:1014-1065)
        const int jr = gy - y_ctb_c;
        int s2 = 7, y1 = 1, y2 = 2;  // Table 46, always with the line-buffer arms
        if (jr == ctb_h_c - 2 || jr == ctb_h_c - 3) { s2 = 10; y1 = y2 = 0; }
        else if (jr == ctb_h_c - 1 || jr == ctb_h_c - 4) { y2 = 1; }
        auto tap = [&](int k, int dx, int dy) {
          const int lim = cclip[k];
          return clampd((int)sC[r + dy][c + dx] - cur, -lim, lim) + clampd((int)sC[r - dy][c - dx] - cur, -lim, lim);
        };
        int sum = ccoef[0] * tap(0, 0, y2);
        sum += ccoef[1] * tap(1, 1, y1);
        sum += ccoef[2] * tap(2, 0, y1);
        sum += ccoef[3] * tap(3, -1, y1);
        sum += ccoef[4] * tap(4, 2, 0);
        sum += ccoef[5] * tap(5, 1, 0);
        v = clampd(cur + ((sum + (1 << (s2 - 1))) >> s2), 0, maxv);
      }
      if (ccf >= 0) {  // §8.8.5.7 CC-ALF (apply_cc_alf_ctb, src/alf.rs:447-523)
        const int yline = (gy - y_ctb_c) * shc;
        const bool lbb = !(gy * shc + ctb >= ph && (ph - y_ctb_c * shc) <= ctb - 4);  // src/alf.rs:484-485
        int yp1 = 1, yp2 = 2;  // Table 47
        if (lbb) {
          if (yline == ctb - 5 || yline == ctb - 4) { yp1 = 0; yp2 = 0; }
          else if (yline == ctb - 6 || yline == ctb - 3) { yp2 = 1; }
        }
        const int lr = gy * shc - (Y0 - 3), lcol = gx * sw - (X0 - 3);
        const int ctr = sL[lr][lcol];
        int sum = cc[0] * ((int)sL[lr - yp1][lcol] - ctr);
        sum += cc[1] * ((int)sL[lr][lcol - 1] - ctr);
        sum += cc[2] * ((int)sL[lr][lcol + 1] - ctr);
        sum += cc[3] * ((int)sL[lr + yp1][lcol - 1] - ctr);
        sum += cc[4] * ((int)sL[lr + yp1][lcol] - ctr);
        sum += cc[5] * ((int)sL[lr + yp1][lcol + 1] - ctr);
        sum += cc[6] * ((int)sL[lr + yp2][lcol] - ctr);
        const int scaled = clampd((sum + 64) >> 7, -half, half - 1);
        const bool suppress = shc == 1 && (yline == ctb - 3 || yline == ctb - 4);
        v = clampd(suppress ? v : v + scaled, 0, maxv);
      }
      CD.s[(int64_t)gy * CD.stride + gx] = (uint16_t)v;
    }
  }
  (void)x_ctb_c;
  (void)ctb_w_c;
}

}  // namespace

int launch_pass2(cudaStream_t st, const Pass2Args &a, bool do_sao, bool do_alf, uint64_t *launches) {
  const unsigned n = (unsigned)(a.tiles_x * a.tiles_y);
  if (n == 0) return H266_OK;
  if (do_sao && do_alf) k_sao_alf<true, true><<<n, NTHREADS, 0, st>>>(a);
  else if (do_sao) k_sao_alf<true, false><<<n, NTHREADS, 0, st>>>(a);
  else if (do_alf) k_sao_alf<false, true><<<n, NTHREADS, 0, st>>>(a);
  else k_sao_alf<false, false><<<n, NTHREADS, 0, st>>>(a);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

}  // namespace h266
