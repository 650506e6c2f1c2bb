// Encoder luma ALF trials (src/alf_enc.rs:185-528): every candidate filter
// set of a CTB evaluated on one staged window, and the per-CTB decision.  The
// chain's SAO / ALF tile pass is in sao_alf3.cu; both use alf_tile.cuh.
#include "alf_tile.cuh"

namespace h266 {
namespace {

using namespace tile;

constexpr int TH = 32;
constexpr int NT = 256;

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
  static constexpr int SLP = SLW;                         // its row pitch
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
  luma_cells<S, NT>(sm.sL, sm.cell);
  __syncthreads();
  luma_classes<W, TH, S, NT>(sm.sL, sm.cell, sm.cls_f, sm.cls_t, Y0, y_ctb, ctb, ph, bd);
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
            hi = __dp2a_hi((int)sum[rr][q][k], (int)f[k], hi);
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

}  // namespace

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

}  // namespace h266
