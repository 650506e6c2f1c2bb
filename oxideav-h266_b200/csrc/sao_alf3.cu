// SAO + ALF + CC-ALF tile pass of the chain (src/sao.rs:389-626, src/alf.rs:
// 220-1143), packed-arithmetic form: the default for BitDepth <= 14, ALF
// coefficients in [-128, 127] and 4:2:0 / 4:0:0 chroma; other inputs use the
// scalar pass in sao_alf.cu.  Like the reference, the pass reads the deblocked
// planes and writes the final planes (its snapshot semantics), and post-SAO
// samples are clamped into the CTB's ALF fetch rectangle (the reference's
// clamped sample()).
//
// One CTA per W x TH luma tile (64 x 64 for CTBs of 64 and 128, 32 x 32 for
// CTBs of 32), never straddling a CTB, so the CTB's parameters, clip
// rectangle and virtual boundary are uniform per tile.  Phases, one barrier
// each:
//  1. the deblocked windows of the three planes, staged by the TMA unit (2-D
//     tensor loads of the tile widened by the halo; out-of-picture samples
//     read as 0 and are never used, as every read is clamped into the clip
//     rectangle) while the CTA resolves the SAO parameters of the 3x3 CTB
//     neighbourhood;
//  2. post-SAO windows of all planes: inside the tile's own CTB and clip
//     rectangle two samples per thread step in packed 16-bit lanes (sign
//     terms by lane-wise clamps, offsets looked up from a signed-byte table
//     with one byte permute), the rest sample by sample;
//  3. luma Laplacian sums per 2x2 cell beside the chroma planes' 5x5 ALF and
//     CC-ALF (a thread per 8 chroma samples of a row, CC-ALF taps as 6 dp2a);
//  4. luma classes, one 4x4 block per thread;
//  5. the 7x7 luma diamond, one block per thread with its 12 taps in
//     registers and each of the 7 rows held as packed words.
#include <atomic>
#include <type_traits>
#include <utility>

#include "alf_tile.cuh"
#include "tma.cuh"

namespace h266 {
namespace {

using namespace tile;

constexpr int NT3 = 256;
constexpr uint64_t kWaitNs = 20000000;  // 20 ms: a tile gives up on its window copies after this

// Tiles whose window copies did not complete within the poll limit (they are
// left unfiltered); read and cleared by pass2_wait_timeouts.
__device__ unsigned int g_wait_timeouts;

template <int W, int TH>
struct Smem3 {
  static constexpr int DLW = W + 16, DLH = TH + 8;          // deblocked luma [X0-8, X1+8) x [Y0-4, Y1+4)
  static constexpr int SLW = W + 8, SLH = TH + 6;           // post-SAO luma [X0-4, X1+4) x [Y0-3, Y1+3)
  static constexpr int CW = W / 2 + 2, CH = TH / 2 + 2;     // 2x2 Laplacian cells
  static constexpr int DCW = W / 2 + 16, DCH = TH / 2 + 6;  // deblocked chroma [x-8, x+8) x [y-3, y+3)
  static constexpr int SCW = W / 2 + 8, SCH = TH / 2 + 4;   // post-SAO chroma [x-4, x+4) x [y-2, y+2)
  // Row pitches of the post-SAO windows: 4 samples past the widths, so that
  // the chroma-phase threads (8 chroma rows of 4 runs per warp) reading luma
  // rows 2 apart, or chroma rows 1 apart, spread over more shared-memory
  // banks; multiples of 4 samples keep the 8-byte row alignment.
  static constexpr int SLP = SLW + 4, SCP = SCW + 4;
  static constexpr int DL_BYTES = DLH * DLW * 2, DC_BYTES = DCH * DCW * 2;
  static constexpr int DC_OFF = (DL_BYTES + 127) & ~127;
  static constexpr int DC_STRIDE = (DC_BYTES + 127) & ~127;
  static constexpr int D_BYTES = DC_OFF + 2 * DC_STRIDE;
  static constexpr int CELL_BYTES = CH * CW * 16;
  static constexpr int U_BYTES = D_BYTES > CELL_BYTES ? D_BYTES : CELL_BYTES;
  // the deblocked windows (TMA destinations); the Laplacian cells reuse the
  // space once the post-SAO windows exist
  alignas(128) uint8_t u[U_BYTES];
  alignas(16) uint16_t sL[SLH * SLP];
  alignas(16) uint16_t sC[2][SCH * SCP];
  uint8_t cls_f[(TH / 4) * (W / 4)], cls_t[(TH / 4) * (W / 4)];
  SaoLocal sao[3][9];
  alignas(8) unsigned long long bar;
  unsigned any_sao;  // bit comp * 9 + n: neighbour n of the 3x3 CTB neighbourhood has SAO for comp
  __device__ uint16_t *dL() { return reinterpret_cast<uint16_t *>(u); }
  __device__ uint16_t *dC(int c) { return reinterpret_cast<uint16_t *>(u + DC_OFF + c * DC_STRIDE); }
  __device__ uint4 *cell() { return reinterpret_cast<uint4 *>(u); }
};

// TMA and mbarrier helpers (tma.cuh); waits give up after kWaitNs.
using namespace tile_dev;

// f(integral_constant<int, 0>) ... f(integral_constant<int, N - 1>): indices as constants
template <class F, int... I>
__device__ __forceinline__ void static_for_impl(F &&f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void static_for(F &&f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// ---------------------------------------------------------------- packed helpers
__device__ __forceinline__ uint32_t ld32(const uint16_t *p) { return *reinterpret_cast<const uint32_t *>(p); }
__device__ __forceinline__ uint2 ld64(const uint16_t *p) { return *reinterpret_cast<const uint2 *>(p); }
__device__ __forceinline__ void st32(uint16_t *p, uint32_t v) { *reinterpret_cast<uint32_t *>(p) = v; }

// Byte permute with sign replication (PTX prmt, default mode: selector bit 3
// copies the sign bit of the selected byte).
__device__ __forceinline__ uint32_t prmt(uint32_t lo, uint32_t hi, uint32_t sel) {
  uint32_t r;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(lo), "r"(hi), "r"(sel));
  return r;
}

// Selector that turns per-lane byte indices (0..7 in each 16-bit lane) into
// the two lanes' sign-extended table bytes.
__device__ __forceinline__ uint32_t lane_sel(uint32_t idx) {
  const uint32_t t = (idx | (idx >> 8)) & 0x0707u;  // lane 0 index in bits 0-2, lane 1 in bits 8-10
  return t | (t << 4) | 0x8080u;
}

// Pair (p[0], p[1]) at any sample offset (odd offsets from two aligned words).
__device__ __forceinline__ uint32_t pair_any(const uint16_t *p, bool odd) {
  return odd ? __byte_perm(ld32(p - 1), ld32(p + 1), 0x5432) : ld32(p);
}

// Per-component state of the packed SAO step: the tile's own CTB parameters.
struct SaoFast {
  int type;          // 0 copy, 1 band, 2 edge
  int nb;            // neighbour offset in the window (edge)
  bool nb_odd;
  uint32_t tlo, thi;  // signed-byte offset table
  uint32_t shift, lane_mask, band_add;  // band: lane index ((c >> shift) - band) & 31
};

__device__ __forceinline__ SaoFast sao_fast(const SaoLocal &p, bool on) {
  SaoFast f;
  f.type = on ? p.type : 0;
  f.nb = p.nb;
  f.nb_odd = (p.nb & 1) != 0;
  f.tlo = p.tlo;
  f.thi = p.thi;
  f.shift = (uint32_t)p.bd_shift;
  const uint32_t m = 0xFFFFu >> p.bd_shift;
  f.lane_mask = m | (m << 16);
  f.band_add = (uint32_t)((32 - p.band) & 31) * 0x00010001u;
  return f;
}

// SAO of the pair at d (window pointer; both samples inside the CTB, the clip
// rectangle and the edge-offset availability rectangle), samples below 2^12.
__device__ __forceinline__ uint32_t sao_pair(const SaoFast &f, const uint16_t *d, uint32_t maxv2) {
  const uint32_t c = ld32(d);
  if (f.type == 0) return c;
  uint32_t off;
  if (f.type == 2) {
    const uint32_t a = pair_any(d + f.nb, f.nb_odd), b = pair_any(d - f.nb, f.nb_odd);
    const uint32_t cb = c | 0x80008000u;
    // lane-wise sign(c - n) + 2 in [1, 3]; the two add to 2 + sign + sign + 2
    const uint32_t sa =
        __viaddmin_s16x2(__viaddmax_s16x2((cb - a) ^ 0x80008000u, 0x00020002u, 0x00010001u), 0u, 0x00030003u);
    const uint32_t sb =
        __viaddmin_s16x2(__viaddmax_s16x2((cb - b) ^ 0x80008000u, 0x00020002u, 0x00010001u), 0u, 0x00030003u);
    off = prmt(f.tlo, f.thi, lane_sel(sa + sb));
  } else {
    const uint32_t k = (((c >> f.shift) & f.lane_mask) + f.band_add) & 0x001F001Fu;
    off = prmt(f.tlo, f.thi, lane_sel(__viaddmin_u16x2(k, 0u, 0x00040004u)));
  }
  return __viaddmin_s16x2(__viaddmax_s16x2(c, off, 0u), 0u, maxv2);
}

// A rectangle of window positions: [x0, x0 + 2 * npx) x [y0, y0 + ny) in
// pairs (fast) or the remaining window samples around it (slow).
struct FastRect {
  int x0, y0, npx, ny;
  uint32_t magic;  // floor(i / npx) = umulhi(i, magic) for the indices used (npx > 1)
  __device__ int row_of(uint32_t i) const { return npx == 1 ? (int)i : (int)__umulhi(i, magic); }
  __device__ int pairs() const { return npx * ny; }
};

__device__ __forceinline__ FastRect fast_rect(int x0, int x1, int y0, int y1) {
  FastRect r;
  x0 = (x0 + 1) & ~1;
  x1 &= ~1;
  r.x0 = x0;
  r.y0 = y0;
  r.npx = x1 > x0 ? (x1 - x0) / 2 : 0;
  r.ny = y1 > y0 ? y1 - y0 : 0;
  if (!r.npx || !r.ny) r.npx = r.ny = 0;
  r.magic = r.npx > 1 ? 0xFFFFFFFFu / (uint32_t)r.npx + 1u : 0u;  // 2^32 / 1 does not fit: row_of
  return r;
}

// The i-th window sample outside the fast rectangle of a WW x WH window whose
// origin is (wx0, wy0): rows above, rows below, then the left and right parts
// of the fast rows.
__device__ __forceinline__ void slow_pos(int i, int wx0, int wy0, int WW, int WH, const FastRect &f, int &x, int &y) {
  const int fy0 = f.ny ? f.y0 : wy0, fy1 = f.ny ? f.y0 + f.ny : wy0;
  const int n_top = WW * (fy0 - wy0), n_bot = WW * (wy0 + WH - fy1);
  if (i < n_top) {
    y = wy0 + i / WW;
    x = wx0 + i % WW;
    return;
  }
  i -= n_top;
  if (i < n_bot) {
    y = fy1 + i / WW;
    x = wx0 + i % WW;
    return;
  }
  i -= n_bot;
  const int lw = f.x0 - wx0, n_left = lw * f.ny;
  if (i < n_left) {
    y = fy0 + i / lw;
    x = wx0 + i % lw;
    return;
  }
  i -= n_left;
  const int rw = wx0 + WW - (f.x0 + 2 * f.npx);
  y = fy0 + i / rw;
  x = f.x0 + 2 * f.npx + i % rw;
}

__device__ __forceinline__ int slow_count(int WW, int WH, const FastRect &f) { return WW * WH - 2 * f.pairs(); }

// Rows of packed words around a run of samples: word k covers samples
// (c0 - 2B + 2k, c0 - 2B + 2k + 1) of the row at p = &row[c0].
template <int NW, int B>
struct Words {
  uint32_t w[NW];
  // pair (p[o], p[o + 1])
  template <int O>
  __device__ __forceinline__ uint32_t pair() const {
    static_assert(O + 2 * B >= 0 && O + 2 * B + 1 < 2 * NW, "pair inside the loaded words");
    if constexpr (((O + 2 * B) & 1) == 0) return w[(O + 2 * B) / 2];
    else return __byte_perm(w[(O + 2 * B - 1) / 2], w[(O + 2 * B + 1) / 2], 0x5432);
  }
};

// Loads words [k0, k1) of a Words<NW, B> at p (p - 2B + 2k0 4-byte aligned;
// 64-bit loads where the address is 8-byte aligned by construction: A8).
template <int NW, int B, bool A8>
__device__ __forceinline__ void load_words(Words<NW, B> &r, const uint16_t *p, int k0, int k1) {
  const uint16_t *q = p - 2 * B;
  // word k starts an 8-byte aligned pair of words
  auto lead = [](int k) { return A8 && (((2 * B) % 4 == 0) == (k % 2 == 0)); };
#pragma unroll
  for (int k = 0; k < NW; ++k) {
    if (k < k0 || k >= k1) continue;
    if (k > k0 && lead(k - 1)) continue;  // loaded with word k - 1
    if (lead(k) && k + 1 < k1) {
      const uint2 v = ld64(q + 2 * k);
      r.w[k] = v.x;
      r.w[k + 1 < NW ? k + 1 : k] = v.y;
    } else {
      r.w[k] = ld32(q + 2 * k);
    }
  }
}

// ---------------------------------------------------------------- the tile
// Tile `tile` of the picture whose parameters are `a` (tensor maps at `maps`).
// PERSIST: the CTA runs many tiles on one barrier, initialised by the caller;
// `phase` is the barrier's next phase and flips with every completed copy.
// Returns false when the window copies did not land in time (the tile is left
// unfiltered and counted; a persistent CTA stops then).
template <int W, int TH, bool DO_SAO, bool DO_ALF, bool GLOBAL_MAPS, bool PERSIST = false>
__device__ __forceinline__ bool sao_alf_tile3(const Pass2Args &a, const Pass2Args *maps, int tile,
                                              uint32_t &phase) {
  using S = Smem3<W, TH>;
  extern __shared__ __align__(128) uint8_t smem_raw[];
  // TMA destinations need 128-byte aligned shared addresses: align the base
  // explicitly (the launch adds 128 bytes)
  S &sm = *reinterpret_cast<S *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
  const int tid = threadIdx.x;
  const int tx = tile % a.tiles_x, ty = tile / a.tiles_x;
  const int X0 = tx * W, Y0 = ty * TH;
  const int bd = a.bit_depth, maxv = (1 << bd) - 1;
  const uint32_t maxv2 = (uint32_t)maxv * 0x00010001u;
  const int log2 = a.ctb_log2, ctb = 1 << log2;
  const int rx = X0 >> log2, ry = Y0 >> log2;
  const int x_ctb = rx << log2, y_ctb = ry << log2;
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
  bool chroma_on[2];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const DPlane &CS = a.src[c + 1];
    chroma_on[c] = a.chroma && CS.w > 0 && CS.h > 0 && xc0 < CS.w && yc0 < CS.h;
  }
  const bool tma = a.tma != 0;

  // ---- (1) deblocked windows (thread 0 starts the copies first, so they
  // overlap the rest of the phase); SAO parameters of the 3x3 CTB neighbourhood
  if (tma && tid == 0) {
    if (!PERSIST) mbar_init(&sm.bar, 1);
    const uint32_t bytes = (a.src[0].w > 0 && a.src[0].h > 0 ? S::DL_BYTES : 0) +
                           (chroma_on[0] ? S::DC_BYTES : 0) + (chroma_on[1] ? S::DC_BYTES : 0);
    if (GLOBAL_MAPS)
      for (int c = 0; c < 3; ++c) tmap_acquire(&maps->tmap[c]);
    // the previous tile's generic accesses of the window space (ordered by the
    // persistent loop's barrier) come before these copies
    if (PERSIST) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&sm.bar, bytes);
    if (a.src[0].w > 0 && a.src[0].h > 0) tma_load_2d(sm.dL(), &maps->tmap[0], X0 - 8, Y0 - 4, &sm.bar);
#pragma unroll
    for (int c = 0; c < 2; ++c)
      if (chroma_on[c]) tma_load_2d(sm.dC(c), &maps->tmap[1 + c], xc0 - 8, yc0 - 3, &sm.bar);
  }
  int my_type = 0;
  if (tid < 27) {
    const int comp = tid / 9, n = tid % 9;
    const int nx = rx + n % 3 - 1, ny = ry + n / 3 - 1;
    SaoLocal &s = sm.sao[comp][n];
    s.type = 0;
    s.nb = 0;
    s.tlo = s.thi = 0;
    s.bd_shift = bd - 5;
    s.band = 0;
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
      my_type = s.type;
    }
  }
  if (tid < 32) {
    const unsigned m = __ballot_sync(0xFFFFFFFFu, my_type != 0);
    if (tid == 0) sm.any_sao = m;
  }
  if (!tma) {
    // windows by 16-byte vector loads (planes whose layout the TMA unit cannot describe)
    auto load = [&](uint16_t *dst, const DPlane &P, int x0, int y0, int WW, int HH) {
      const bool vec = x0 >= 0 && x0 + WW <= P.w && (x0 & 7) == 0 && ((uintptr_t)P.s & 15) == 0 && (P.stride & 7) == 0;
      if (vec) {
        const int NV = WW / 8;
        for (int i = tid; i < HH * NV; i += NT3) {
          const int r = i / NV, c = (i - r * NV) * 8;
          const int gy = clampd(y0 + r, 0, P.h - 1);
          *reinterpret_cast<uint4 *>(dst + r * WW + c) =
              *reinterpret_cast<const uint4 *>(P.s + (int64_t)gy * P.stride + x0 + c);
        }
      } else {
        for (int i = tid; i < HH * WW; i += NT3) {
          const int r = i / WW, c = i - r * WW;
          const int gx = clampd(x0 + c, 0, P.w - 1), gy = clampd(y0 + r, 0, P.h - 1);
          dst[i] = P.s[(int64_t)gy * P.stride + gx];
        }
      }
    };
    if (a.src[0].w > 0 && a.src[0].h > 0) load(sm.dL(), a.src[0], X0 - 8, Y0 - 4, S::DLW, S::DLH);
#pragma unroll
    for (int c = 0; c < 2; ++c)
      if (chroma_on[c]) load(sm.dC(c), a.src[c + 1], xc0 - 8, yc0 - 3, S::DCW, S::DCH);
  }
  __syncthreads();  // SAO parameters, the barrier's initialisation (or the vector-loaded windows)

  // geometry of the packed SAO rectangles while the copies are in flight
  const unsigned any = sm.any_sao;
  const bool sao_on[3] = {DO_SAO && (any & 0x1FFu) != 0, DO_SAO && ((any >> 9) & 0x1FFu) != 0,
                          DO_SAO && ((any >> 18) & 0x1FFu) != 0};
  // packed SAO: offsets as signed bytes, samples below 2^12 (a plain copy has no such limit)
  const bool fast_ok[3] = {!sao_on[0] || (a.sao_i8 && bd <= 12), !sao_on[1] || (a.sao_i8 && bd <= 12),
                           !sao_on[2] || (a.sao_i8 && bd <= 12)};
  const int crx0 = rect[0] / 2, cry0 = rect[1] / 2, crx1 = (rect[2] + 1) / 2, cry1 = (rect[3] + 1) / 2;
  FastRect fr[3];
  {
    // luma: inside the own CTB and one sample inside the clip rectangle when any
    // SAO is on (edge offset then sees both neighbours); else the clip rectangle
    const bool s = sao_on[0];
    fr[0] = fast_ok[0] ? fast_rect(max(X0 - 4, s ? max(x_ctb, rx0 + 1) : rx0),
                                min(X0 + W + 4, s ? min(x_ctb + ctb, rx1 - 1) : rx1),
                                max(Y0 - 3, s ? max(y_ctb, ry0 + 1) : ry0),
                                min(Y0 + TH + 3, s ? min(y_ctb + ctb, ry1 - 1) : ry1))
                    : fast_rect(0, 0, 0, 0);
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
      const DPlane &CS = a.src[cc + 1];
      const int cx0 = max(crx0, 0), cy0 = max(cry0, 0), cx1 = min(crx1, CS.w), cy1 = min(cry1, CS.h);
      const bool t = sao_on[cc + 1];
      const int cxs = x_ctb / 2, cys = y_ctb / 2, cc_ctb = ctb / 2;
      fr[cc + 1] = (fast_ok[cc + 1] && chroma_on[cc])
                       ? fast_rect(max(xc0 - 4, t ? max(cxs, cx0 + 1) : cx0),
                                   min(xc0 + TWC + 4, t ? min(cxs + cc_ctb, cx1 - 1) : cx1),
                                   max(yc0 - 2, t ? max(cys, cy0 + 1) : cy0),
                                   min(yc0 + THC + 2, t ? min(cys + cc_ctb, cy1 - 1) : cy1))
                       : fast_rect(0, 0, 0, 0);
    }
  }
  if (tma) {
    bool ok = mbar_wait_bounded(&sm.bar, phase, kWaitNs);
    ok = __syncthreads_and(ok);
    if (!ok) {  // the copies did not land: count the tile, let them finish (bounded), leave it unfiltered
      if (tid == 0) atomicAdd(&g_wait_timeouts, 1u);
      mbar_wait_bounded(&sm.bar, phase, kWaitNs);
      return false;
    }
    phase ^= 1u;
  }

  // ---- (2) post-SAO windows, clamped into the fetch rectangle
  const SaoFast fs[3] = {sao_fast(sm.sao[0][4], sao_on[0]), sao_fast(sm.sao[1][4], sao_on[1]),
                         sao_fast(sm.sao[2][4], sao_on[2])};
  {
    const int nf0 = fr[0].pairs(), nf1 = chroma_on[0] ? fr[1].pairs() : 0, nf2 = chroma_on[1] ? fr[2].pairs() : 0;
    const uint16_t *dL = sm.dL();
    for (int i = tid; i < nf0 + nf1 + nf2; i += NT3) {
      if (i < nf0) {
        const FastRect &f = fr[0];
        const int r = f.row_of((uint32_t)i), x = f.x0 + 2 * (i - r * f.npx), y = f.y0 + r;
        const uint16_t *d = dL + (y - (Y0 - 4)) * S::DLW + (x - (X0 - 8));
        st32(&sm.sL[(y - (Y0 - 3)) * S::SLP + (x - (X0 - 4))], sao_pair(fs[0], d, maxv2));
      } else {
        const int cc = i < nf0 + nf1 ? 0 : 1;
        const int j = i - nf0 - (cc ? nf1 : 0);
        const FastRect &f = fr[1 + cc];
        const int r = f.row_of((uint32_t)j), x = f.x0 + 2 * (j - r * f.npx), y = f.y0 + r;
        const uint16_t *d = sm.dC(cc) + (y - (yc0 - 3)) * S::DCW + (x - (xc0 - 8));
        st32(&sm.sC[cc][(y - (yc0 - 2)) * S::SCP + (x - (xc0 - 4))], sao_pair(fs[1 + cc], d, maxv2));
      }
    }
    // the rest sample by sample: neighbouring CTBs, clamped positions, edges of the clip rectangle
    const int ns0 = slow_count(S::SLW, S::SLH, fr[0]);
    const int ns1 = chroma_on[0] ? slow_count(S::SCW, S::SCH, fr[1]) : 0;
    const int ns2 = chroma_on[1] ? slow_count(S::SCW, S::SCH, fr[2]) : 0;
    for (int i = tid; i < ns0 + ns1 + ns2; i += NT3) {
      int x, y;
      if (i < ns0) {
        slow_pos(i, X0 - 4, Y0 - 3, S::SLW, S::SLH, fr[0], x, y);
        const int ax = clampd(x, rx0, rx1 - 1), ay = clampd(y, ry0, ry1 - 1);
        const uint16_t *d = &dL[(ay - (Y0 - 4)) * S::DLW + ax - (X0 - 8)];
        int v = *d;
        if (sao_on[0]) {
          const SaoLocal &p = sm.sao[0][((ay >> log2) - ry + 1) * 3 + ((ax >> log2) - rx + 1)];
          if (p.type) v = sao_one(p, ax, ay, maxv, d);
        }
        sm.sL[(y - (Y0 - 3)) * S::SLP + (x - (X0 - 4))] = (uint16_t)v;
      } else {
        const int cc = i < ns0 + ns1 ? 0 : 1;
        const int j = i - ns0 - (cc ? ns1 : 0);
        slow_pos(j, xc0 - 4, yc0 - 2, S::SCW, S::SCH, fr[1 + cc], x, y);
        const DPlane &CS = a.src[cc + 1];
        const int cx0 = max(crx0, 0), cy0 = max(cry0, 0), cx1 = min(crx1, CS.w), cy1 = min(cry1, CS.h);
        const int ax = clampd(x, cx0, cx1 - 1), ay = clampd(y, cy0, cy1 - 1);
        const uint16_t *d = sm.dC(cc) + (ay - (yc0 - 3)) * S::DCW + ax - (xc0 - 8);
        int v = *d;
        if (sao_on[1 + cc]) {
          const SaoLocal &p = sm.sao[cc + 1][(((ay * 2) >> log2) - ry + 1) * 3 + (((ax * 2) >> log2) - rx + 1)];
          if (p.type) v = sao_one(p, ax, ay, maxv, d);
        }
        sm.sC[cc][(y - (yc0 - 2)) * S::SCP + (x - (xc0 - 4))] = (uint16_t)v;
      }
    }
  }
  __syncthreads();

  // ---- (3) luma Laplacian sums per 2x2 cell (into the dead deblocked windows); chroma ALF / CC-ALF
  const bool luma_alf = DO_ALF && me && me->luma_set >= 0;
  if (luma_alf) luma_cells<S, NT3>(sm.sL, sm.cell());
  {
    // thread -> (plane, row, run of SPT samples)
    constexpr int SPT = TWC * THC / (NT3 / 2);  // 8 (64 x 64 tiles) or 2 (32 x 32)
    constexpr int NP = SPT / 2;                 // pairs per thread
    constexpr int RPR = TWC / SPT;              // threads per chroma row
    const int cc = tid / (NT3 / 2), t = tid % (NT3 / 2);
    const int jj = t / RPR, i0 = (t % RPR) * SPT;
    const DPlane &CD = a.dst[cc + 1];
    const int gy = yc0 + jj, gx = xc0 + i0;
    if (chroma_on[cc] && gy < CD.h && gx < CD.w) {
      const int cf = (DO_ALF && me) ? me->chroma_filt[cc] : -1;
      const int ccf = (DO_ALF && me) ? me->cc_filt[cc] : -1;
      const int ctb_c = ctb / 2, y_ctb_c = y_ctb / 2;
      const int c0 = i0 + 4;
      const uint16_t *R0 = &sm.sC[cc][(jj + 2) * S::SCP + c0];
      int v[SPT];
      {
        Words<NP + 2, 1> w0;
        load_words<NP + 2, 1, (NP > 1)>(w0, R0, 1, NP + 1);
#pragma unroll
        for (int q = 0; q < NP; ++q) {
          const uint32_t cur = w0.w[1 + q];
          v[2 * q] = (int)(cur & 0xFFFF);
          v[2 * q + 1] = (int)(cur >> 16);
        }
      }
      if (cf >= 0) {  // 5x5 diamond (src/alf.rs:1014-1065, Table 46 line-buffer arms always applied)
        const int jr = gy - y_ctb_c;
        int s2 = 7, y1 = 1, y2 = 2;
        if (jr == ctb_c - 2 || jr == ctb_c - 3) { s2 = 10; y1 = y2 = 0; }
        else if (jr == ctb_c - 1 || jr == ctb_c - 4) { y2 = 1; }
        const uint32_t *ct = a.tables.chroma_packed + min(cf, 7) * 18;
        uint32_t c2[6], nc2[6], f[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          c2[k] = ct[3 * k];
          nc2[k] = ct[3 * k + 1];
          f[k] = ct[3 * k + 2];
        }
        int acc[SPT];
#pragma unroll
        for (int k = 0; k < SPT; ++k) acc[k] = 0;
        uint32_t ncur[NP];
        Words<NP + 2, 1> r0, ra, rb;
        load_words<NP + 2, 1, (NP > 1)>(r0, R0, 0, NP + 2);
#pragma unroll
        for (int q = 0; q < NP; ++q) ncur[q] = neg2(r0.w[1 + q]);
        auto tap = [&](const Words<NP + 2, 1> &up, const Words<NP + 2, 1> &dn, auto dx, int k) {
          constexpr int DX = decltype(dx)::value;
          static_for<NP>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            const uint32_t x = clipd(up.template pair<DX + 2 * q>(), ncur[q], c2[k], nc2[k]);
            const uint32_t y = clipd(dn.template pair<-DX + 2 * q>(), ncur[q], c2[k], nc2[k]);
            const uint32_t s = add2(x, y);
            acc[2 * q] = __dp2a_lo((int)s, (int)f[k], acc[2 * q]);
            acc[2 * q + 1] = __dp2a_hi((int)s, (int)f[k], acc[2 * q + 1]);
          });
        };
        using I0 = std::integral_constant<int, 0>;
        using I1 = std::integral_constant<int, 1>;
        using Im1 = std::integral_constant<int, -1>;
        using I2 = std::integral_constant<int, 2>;
        load_words<NP + 2, 1, (NP > 1)>(ra, R0 + y2 * S::SCP, 1, NP + 1);
        load_words<NP + 2, 1, (NP > 1)>(rb, R0 - y2 * S::SCP, 1, NP + 1);
        tap(ra, rb, I0{}, 0);
        load_words<NP + 2, 1, (NP > 1)>(ra, R0 + y1 * S::SCP, 0, NP + 2);
        load_words<NP + 2, 1, (NP > 1)>(rb, R0 - y1 * S::SCP, 0, NP + 2);
        tap(ra, rb, I1{}, 1);
        tap(ra, rb, I0{}, 2);
        tap(ra, rb, Im1{}, 3);
        tap(r0, r0, I2{}, 4);
        tap(r0, r0, I1{}, 5);
        const int round = 1 << (s2 - 1);
#pragma unroll
        for (int k = 0; k < SPT; ++k) v[k] = clampd(v[k] + ((acc[k] + round) >> s2), 0, maxv);
      }
      if (ccf >= 0) {  // CC-ALF from post-SAO luma (Table 47, src/alf.rs:447-523)
        const int *cc_k = a.tables.cc_coeff[cc][ccf];
        auto b8 = [](int x) { return (uint32_t)(x & 0xFF); };
        // taps 0..6 at (0,-yP1), (-1,0), (+1,0), (-1,yP1), (0,yP1), (+1,yP1), (0,yP2) as dp2a byte pairs
        const uint32_t k1 = b8(cc_k[0]) | b8(cc_k[1]) << 24;
        const uint32_t k2 = b8(cc_k[2]) << 8 | b8(cc_k[3]) << 24;
        const uint32_t k3 = b8(cc_k[4]) | b8(cc_k[5]) << 8 | b8(cc_k[6]) << 16;
        const int csum = cc_k[0] + cc_k[1] + cc_k[2] + cc_k[3] + cc_k[4] + cc_k[5] + cc_k[6];
        const int half = 1 << (bd - 1);
        const int yline = (gy - y_ctb_c) * 2;
        const bool lbb = !(gy * 2 + ctb >= ph && (ph - y_ctb) <= ctb - 4);
        int yp1 = 1, yp2 = 2;
        if (lbb) {
          if (yline == ctb - 5 || yline == ctb - 4) { yp1 = 0; yp2 = 0; }
          else if (yline == ctb - 6 || yline == ctb - 3) { yp2 = 1; }
        }
        // luma words of the run: word k = samples (2 i0 + 2 + 2k, +1) of a window row (col 2 i0 + 4 = luma x of i0)
        const uint16_t *L0 = &sm.sL[(2 * jj + 3) * S::SLP + 2 * i0 + 4];
        // 8-byte loads for word pairs (k, k + 1), k odd (L0 is 8-byte aligned when SPT > 2)
        constexpr int LW = SPT + 1;
        Words<LW, 1> wt, wm, wb, w2;
        load_words<LW, 1, (SPT > 2)>(wt, L0 - yp1 * S::SLP, 0, LW);
        load_words<LW, 1, (SPT > 2)>(wm, L0, 0, LW);
        load_words<LW, 1, (SPT > 2)>(wb, L0 + yp1 * S::SLP, 0, LW);
        load_words<LW, 1, (SPT > 2)>(w2, L0 + yp2 * S::SLP, 0, LW);
#pragma unroll
        for (int k = 0; k < SPT; ++k) {
          // chroma sample k: luma (2k - 1, 2k) in word k, (2k, 2k + 1) in word k + 1
          int s = __dp2a_lo((int)wt.w[k + 1], (int)k1, 0);
          s = __dp2a_hi((int)wm.w[k], (int)k1, s);
          s = __dp2a_lo((int)wm.w[k + 1], (int)k2, s);
          s = __dp2a_hi((int)wb.w[k], (int)k2, s);
          s = __dp2a_lo((int)wb.w[k + 1], (int)k3, s);
          s = __dp2a_hi((int)w2.w[k + 1], (int)k3, s);
          const int ctr = (int)(wm.w[k + 1] & 0xFFFF);
          s -= ctr * csum;
          v[k] = clampd(v[k] + clampd((s + 64) >> 7, -half, half - 1), 0, maxv);
        }
      }
      uint16_t *out = CD.s + (int64_t)gy * CD.stride + gx;
      const bool vec = gx + SPT <= CD.w && ((uintptr_t)out & (2 * SPT - 1)) == 0;
      if (vec && SPT == 8) {
        uint4 o;
        o.x = (uint32_t)v[0] | (uint32_t)v[1] << 16;
        o.y = (uint32_t)v[2] | (uint32_t)v[3] << 16;
        o.z = (uint32_t)v[4] | (uint32_t)v[5] << 16;
        o.w = (uint32_t)v[6 % SPT] | (uint32_t)v[7 % SPT] << 16;
        *reinterpret_cast<uint4 *>(out) = o;
      } else if (vec && SPT == 4) {
        *reinterpret_cast<uint2 *>(out) = make_uint2((uint32_t)v[0] | (uint32_t)v[1 % SPT] << 16,
                                                     (uint32_t)v[2 % SPT] | (uint32_t)v[3 % SPT] << 16);
      } else if (vec && SPT == 2) {
        *reinterpret_cast<uint32_t *>(out) = (uint32_t)v[0] | (uint32_t)v[1 % SPT] << 16;
      } else {
#pragma unroll
        for (int k = 0; k < SPT; ++k)
          if (gx + k < CD.w) out[k] = (uint16_t)v[k];
      }
    }
  }
  const DPlane LD = a.dst[0];
  if (!luma_alf) {
    // the post-SAO tile as it is, 4 samples per store
    for (int p = tid; p < TH * W / 4; p += NT3) {
      const int j = p / (W / 4), i = (p % (W / 4)) * 4;
      const int gx = X0 + i, gy = Y0 + j;
      if (gy >= LD.h || gx >= LD.w) continue;
      const uint2 v = ld64(&sm.sL[(j + 3) * S::SLP + i + 4]);
      uint16_t *out = LD.s + (int64_t)gy * LD.stride + gx;
      if (gx + 4 <= LD.w && ((uintptr_t)out & 7) == 0) {
        *reinterpret_cast<uint2 *>(out) = v;
      } else {
        const uint16_t s4[4] = {(uint16_t)(v.x & 0xFFFF), (uint16_t)(v.x >> 16), (uint16_t)(v.y & 0xFFFF),
                                (uint16_t)(v.y >> 16)};
        for (int k = 0; k < 4 && gx + k < LD.w; ++k) out[k] = s4[k];
      }
    }
    return true;
  }
  __syncthreads();

  // ---- (4) classes
  luma_classes<W, TH, S, NT3>(sm.sL, sm.cell(), sm.cls_f, sm.cls_t, Y0, y_ctb, ctb, ph, bd);
  __syncthreads();

  // ---- (5) 7x7 diamond: every thread keeps one block's taps and filters RPT of its 4-sample runs
  constexpr int RUNS = TH * W / 4;
  constexpr int RPT = RUNS / NT3;  // runs per thread: 4 (64 x 64) or 1 (32 x 32)
  constexpr int TPB = 4 / RPT;     // threads per 4x4 block
  const int b = tid / TPB;
  const int bx = b % (W / 4), by = b / (W / 4);
  const uint32_t *tab = a.tables.luma_packed + ((size_t)me->luma_set * 100 + sm.cls_f[b] * 4 + sm.cls_t[b]) * 36;
  // clip values and coefficients in registers (the negated clips are formed per use: fewer live registers)
  uint32_t c2[12], f[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    c2[k] = __ldg(tab + 3 * k);
    f[k] = __ldg(tab + 3 * k + 2);
  }
  const int gx = X0 + 4 * bx;
#pragma unroll 1
  for (int rr = 0; rr < RPT; ++rr) {
    const int j = 4 * by + (tid % TPB) * RPT + rr;  // tile row
    const int gy = Y0 + j;
    if (gy >= LD.h || gx >= LD.w) continue;
    int shift, y1, y2, y3;
    table45(gy - y_ctb, ctb, shift, y1, y2, y3);
    const uint16_t *R0 = &sm.sL[(j + 3) * S::SLP + 4 * bx + 4];
    int acc[4] = {0, 0, 0, 0};
    uint32_t cur[2], ncur[2];
    // words k of a row: samples (c0 - 4 + 2k, +1), c0 = the run's first sample
    Words<6, 2> ru, rd;
    auto tap = [&](const Words<6, 2> &up, const Words<6, 2> &dn, auto dx, int k) {
      constexpr int DX = decltype(dx)::value;
      const uint32_t nc = neg2(c2[k]);
      static_for<2>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        const uint32_t x = clipd(up.template pair<DX + 2 * q>(), ncur[q], c2[k], nc);
        const uint32_t y = clipd(dn.template pair<-DX + 2 * q>(), ncur[q], c2[k], nc);
        const uint32_t s = add2(x, y);
        acc[2 * q] = __dp2a_lo((int)s, (int)f[k], acc[2 * q]);
        acc[2 * q + 1] = __dp2a_hi((int)s, (int)f[k], acc[2 * q + 1]);
      });
    };
    using I0 = std::integral_constant<int, 0>;
    using I1 = std::integral_constant<int, 1>;
    using Im1 = std::integral_constant<int, -1>;
    using I2 = std::integral_constant<int, 2>;
    using Im2 = std::integral_constant<int, -2>;
    using I3 = std::integral_constant<int, 3>;
    load_words<6, 2, true>(ru, R0, 0, 6);  // the run's own row
    cur[0] = ru.w[2];
    cur[1] = ru.w[3];
    ncur[0] = neg2(cur[0]);
    ncur[1] = neg2(cur[1]);
    tap(ru, ru, I3{}, 9);
    tap(ru, ru, I2{}, 10);
    tap(ru, ru, I1{}, 11);
    load_words<6, 2, true>(ru, R0 + y3 * S::SLP, 2, 4);
    load_words<6, 2, true>(rd, R0 - y3 * S::SLP, 2, 4);
    tap(ru, rd, I0{}, 0);
    load_words<6, 2, true>(ru, R0 + y2 * S::SLP, 1, 5);
    load_words<6, 2, true>(rd, R0 - y2 * S::SLP, 1, 5);
    tap(ru, rd, I1{}, 1);
    tap(ru, rd, I0{}, 2);
    tap(ru, rd, Im1{}, 3);
    load_words<6, 2, true>(ru, R0 + y1 * S::SLP, 1, 5);
    load_words<6, 2, true>(rd, R0 - y1 * S::SLP, 1, 5);
    tap(ru, rd, I2{}, 4);
    tap(ru, rd, I1{}, 5);
    tap(ru, rd, I0{}, 6);
    tap(ru, rd, Im1{}, 7);
    tap(ru, rd, Im2{}, 8);
    const int round = 1 << (shift - 1);
    int o[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const int cv = (int)((cur[p >> 1] >> ((p & 1) * 16)) & 0xFFFF);
      o[p] = clampd(cv + ((acc[p] + round) >> shift), 0, maxv);
    }
    uint16_t *out = LD.s + (int64_t)gy * LD.stride + gx;
    if (gx + 4 <= LD.w && ((uintptr_t)out & 7) == 0) {
      *reinterpret_cast<uint2 *>(out) =
          make_uint2((uint32_t)o[0] | (uint32_t)o[1] << 16, (uint32_t)o[2] | (uint32_t)o[3] << 16);
    } else {
      for (int p = 0; p < 4 && gx + p < LD.w; ++p) out[p] = (uint16_t)o[p];
    }
  }
  return true;
}

template <int W, int TH, bool DO_SAO, bool DO_ALF>
__global__ void __launch_bounds__(NT3, 4) k_sao_alf_tiles(const __grid_constant__ Pass2Args a) {
  uint32_t phase = 0;
  sao_alf_tile3<W, TH, DO_SAO, DO_ALF, false>(a, &a, blockIdx.x, phase);
}

// Many pictures in one grid: CTAs [first[i], first[i + 1]) are the tiles of
// picture i, whose parameters (and tensor maps) are args[i].
template <int W, int TH, bool DO_SAO, bool DO_ALF>
__global__ void __launch_bounds__(NT3, 4) k_sao_alf_tiles_batch(const Pass2Args *__restrict__ args,
                                                                const uint32_t *__restrict__ first, int n) {
  __shared__ Pass2Args s_args;  // the picture's parameters, read once per CTA
  int lo = 0, hi = n;            // first[lo] <= blockIdx.x < first[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (first[mid] <= blockIdx.x) lo = mid;
    else hi = mid;
  }
  static_assert(sizeof(Pass2Args) % 16 == 0, "vector copy");
  const uint4 *src = reinterpret_cast<const uint4 *>(args + lo);
  uint4 *dst = reinterpret_cast<uint4 *>(&s_args);
  for (int i = threadIdx.x; i < (int)(sizeof(Pass2Args) / 16); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  uint32_t phase = 0;
  sao_alf_tile3<W, TH, DO_SAO, DO_ALF, true>(s_args, args + lo, (int)(blockIdx.x - first[lo]), phase);
}

// Persistent form of the batched launch: a fixed grid (a chosen number of
// CTAs per SM) drains a device queue of (picture, tile) items -- `queue`
// counts the items handed out (zero at launch) and items [first[i],
// first[i + 1]) are picture i's tiles.  Every CTA keeps one barrier over its
// tiles and reloads the picture's parameters only when the picture changes.
// The queue only ever grows and no CTA waits for another, so the launch ends
// once every item has been taken.
template <int W, int TH, bool DO_SAO, bool DO_ALF>
__global__ void __launch_bounds__(NT3, 4) k_sao_alf_tiles_queue(const Pass2Args *__restrict__ args,
                                                                const uint32_t *__restrict__ first, int n,
                                                                uint32_t total, uint32_t *__restrict__ queue) {
  using S = Smem3<W, TH>;
  extern __shared__ __align__(128) uint8_t smem_raw[];
  S &sm = *reinterpret_cast<S *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
  __shared__ Pass2Args s_args;
  __shared__ uint32_t s_item;
  if (threadIdx.x == 0) mbar_init(&sm.bar, 1);
  uint32_t phase = 0;
  int cur = -1;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(queue, 1u);
    __syncthreads();  // s_item; the previous tile's last reads of s_args and the windows
    const uint32_t t = s_item;
    if (t >= total) break;
    int lo = 0, hi = n;  // first[lo] <= t < first[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (first[mid] <= t) lo = mid;
      else hi = mid;
    }
    if (lo != cur) {
      const uint4 *src = reinterpret_cast<const uint4 *>(args + lo);
      uint4 *dst = reinterpret_cast<uint4 *>(&s_args);
      for (int i = threadIdx.x; i < (int)(sizeof(Pass2Args) / 16); i += blockDim.x) dst[i] = src[i];
      cur = lo;
    }
    __syncthreads();
    if (!sao_alf_tile3<W, TH, DO_SAO, DO_ALF, true, true>(s_args, args + lo, (int)(t - first[lo]), phase)) break;
    __syncthreads();  // every thread is done with this tile before thread 0 takes the next item
  }
}

template <int W, int TH>
constexpr size_t smem3() {
  return sizeof(Smem3<W, TH>) + 128;
}

// W x TH of a picture's tiles: 64 x 64 (or 64 x 32 by tuning) for CTBs of 64
// and 128, 32 x 32 for 32.
inline int tile_w(int log2) { return log2 >= 6 ? 64 : 32; }
inline int tile_h(const Pass2Args &a) { return tile_w(a.ctb_log2) == 64 && a.tile_h == 32 ? 32 : tile_w(a.ctb_log2); }

// Once per kernel and device: the largest shared-memory carveout, so that four
// CTAs of the tile kernel fit on an SM.
template <class K>
int prepare_kernel(K kern, size_t shm) {
  static_assert(sizeof(Smem3<64, 64>) + 128 + sizeof(Pass2Args) <= 48 * 1024, "default shared-memory limit of a CTA");
  static std::atomic<uint64_t> done{0};
  int dev = 0;
  H266_CUDA(cudaGetDevice(&dev));
  const uint64_t bit = 1ull << (dev & 63);
  if (!(done.load(std::memory_order_relaxed) & bit)) {
    H266_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    done.fetch_or(bit);
  }
  (void)shm;
  return H266_OK;
}

// Host-side driver API entry point for the tensor-map encoder (no libcuda link).
using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_fn() {
  static EncodeTiled fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}

bool encode_plane(CUtensorMap *m, const DPlane &p, int box_w, int box_h) {
  const EncodeTiled enc = encode_fn();
  if (!enc || !p.s || p.w <= 0 || p.h <= 0) return false;
  if (((uintptr_t)p.s & 15) != 0 || (p.stride * 2) % 16 != 0 || p.stride < p.w) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)p.w, (cuuint64_t)p.h};
  const cuuint64_t strides[1] = {(cuuint64_t)p.stride * 2};
  const cuuint32_t box[2] = {(cuuint32_t)box_w, (cuuint32_t)box_h};
  const cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, p.s, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

bool encode_plane_map(CUtensorMap *m, const DPlane &p, int box_w, int box_h) { return encode_plane(m, p, box_w, box_h); }

namespace {

template <int W, int TH>
void maps_for(Pass2Args &a) {
  using S = Smem3<W, TH>;
  bool ok = encode_plane(&a.tmap[0], a.src[0], S::DLW, S::DLH) || a.src[0].w <= 0 || a.src[0].h <= 0;
  for (int c = 1; c < 3 && ok; ++c)
    if (a.chroma && a.src[c].w > 0 && a.src[c].h > 0) ok = encode_plane(&a.tmap[c], a.src[c], S::DCW, S::DCH);
  a.tma = ok ? 1 : 0;
}

template <int W, int TH>
int launch_one(cudaStream_t st, const Pass2Args &in, bool do_sao, bool do_alf) {
  Pass2Args a = in;
  a.tiles_x = (a.ext_w + W - 1) / W;
  a.tiles_y = (a.ext_h + TH - 1) / TH;
  const unsigned n = (unsigned)(a.tiles_x * a.tiles_y);
  const size_t shm = smem3<W, TH>();
  auto go = [&](auto kern) -> int {
    H266_TRY(prepare_kernel(kern, shm));
    kern<<<n, NT3, shm, st>>>(a);
    H266_CUDA(cudaGetLastError());
    return H266_OK;
  };
  if (do_sao && do_alf) return go(k_sao_alf_tiles<W, TH, true, true>);
  if (do_sao) return go(k_sao_alf_tiles<W, TH, true, false>);
  if (do_alf) return go(k_sao_alf_tiles<W, TH, false, true>);
  return go(k_sao_alf_tiles<W, TH, false, false>);
}

}  // namespace

void pass2_tma_maps(Pass2Args &a) {
  if (tile_w(a.ctb_log2) == 32) maps_for<32, 32>(a);
  else if (tile_h(a) == 32) maps_for<64, 32>(a);
  else maps_for<64, 64>(a);
}

int pass2_wait_timeouts(uint32_t *count) {
  unsigned int v = 0, zero = 0;
  H266_CUDA(cudaMemcpyFromSymbol(&v, g_wait_timeouts, sizeof v));
  if (v) H266_CUDA(cudaMemcpyToSymbol(g_wait_timeouts, &zero, sizeof zero));
  *count = v;
  return H266_OK;
}

int pass2_packed_variant(Pass2Args &a, bool do_sao, bool do_alf, uint32_t *ctas) {
  const int W = tile_w(a.ctb_log2), TH = tile_h(a);
  a.tiles_x = (a.ext_w + W - 1) / W;
  a.tiles_y = (a.ext_h + TH - 1) / TH;
  *ctas = a.ext_w > 0 && a.ext_h > 0 ? (uint32_t)(a.tiles_x * a.tiles_y) : 0;
  return (W == 32 ? 0 : (TH == 64 ? 8 : 4)) + (do_sao ? 2 : 0) + (do_alf ? 1 : 0);
}

namespace {
int sm_count() {
  static std::atomic<int> cached{0};
  int v = cached.load();
  if (!v) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      v = 148;
    cached.store(v);
  }
  return v;
}

template <int W, int TH, bool DO_SAO, bool DO_ALF>
int launch_variant(cudaStream_t st, const Pass2Args *d_args, const uint32_t *d_first, int n, uint32_t ctas, int cps,
                   uint32_t *d_queue) {
  const size_t shm = smem3<W, TH>();
  if (cps > 0 && d_queue) {
    auto kern = k_sao_alf_tiles_queue<W, TH, DO_SAO, DO_ALF>;
    H266_TRY(prepare_kernel(kern, shm));
    const uint32_t grid = std::min<uint32_t>(ctas, (uint32_t)(sm_count() * cps));
    kern<<<grid, NT3, shm, st>>>(d_args, d_first, n, ctas, d_queue);
  } else {
    auto kern = k_sao_alf_tiles_batch<W, TH, DO_SAO, DO_ALF>;
    H266_TRY(prepare_kernel(kern, shm));
    kern<<<ctas, NT3, shm, st>>>(d_args, d_first, n);
  }
  H266_CUDA(cudaGetLastError());
  return H266_OK;
}
}  // namespace

int launch_pass2_packed_batch(cudaStream_t st, int variant, const Pass2Args *d_args, const uint32_t *d_first, int n,
                              uint32_t ctas, int ctas_per_sm, uint32_t *d_queue, uint64_t *launches) {
  if (!ctas || n <= 0) return H266_OK;
  int rc;
  const int c = ctas_per_sm;
  switch (variant) {
    case 11: rc = launch_variant<64, 64, true, true>(st, d_args, d_first, n, ctas, c, d_queue); break;
    case 10: rc = launch_variant<64, 64, true, false>(st, d_args, d_first, n, ctas, c, d_queue); break;
    case 9: rc = launch_variant<64, 64, false, true>(st, d_args, d_first, n, ctas, c, d_queue); break;
    case 8: rc = launch_variant<64, 64, false, false>(st, d_args, d_first, n, ctas, c, d_queue); break;
    case 7: rc = launch_variant<64, 32, true, true>(st, d_args, d_first, n, ctas, c, d_queue); break;
    case 6: rc = launch_variant<64, 32, true, false>(st, d_args, d_first, n, ctas, c, d_queue); break;
    case 5: rc = launch_variant<64, 32, false, true>(st, d_args, d_first, n, ctas, c, d_queue); break;
    case 4: rc = launch_variant<64, 32, false, false>(st, d_args, d_first, n, ctas, c, d_queue); break;
    case 3: rc = launch_variant<32, 32, true, true>(st, d_args, d_first, n, ctas, c, d_queue); break;
    case 2: rc = launch_variant<32, 32, true, false>(st, d_args, d_first, n, ctas, c, d_queue); break;
    case 1: rc = launch_variant<32, 32, false, true>(st, d_args, d_first, n, ctas, c, d_queue); break;
    default: rc = launch_variant<32, 32, false, false>(st, d_args, d_first, n, ctas, c, d_queue); break;
  }
  if (rc == H266_OK) ++*launches;
  return rc;
}

int launch_pass2_packed(cudaStream_t st, const Pass2Args &a, bool do_sao, bool do_alf, uint64_t *launches) {
  if (a.ext_w <= 0 || a.ext_h <= 0) return H266_OK;
  const int rc = tile_w(a.ctb_log2) == 64 ? (tile_h(a) == 32 ? launch_one<64, 32>(st, a, do_sao, do_alf)
                                                              : launch_one<64, 64>(st, a, do_sao, do_alf))
                                          : launch_one<32, 32>(st, a, do_sao, do_alf);
  if (rc == H266_OK) ++*launches;
  return rc;
}

}  // namespace h266
