// Encoder SAO decision (src/sao_enc.rs:44-487, sao_decide_picture): per CTB
// and component the band-offset and edge-offset statistics (count and sum of
// src - rec per band / per edge category of each class) gathered on the GPU,
// then the crate's decision arithmetic per CTB on the GPU.
//
// k_sao_stats: one CTA per (CTB, component, 16-row slice); a warp per row,
// 32 columns per step (all lanes step together, so the peer groups of
// __match_any_sync come from a full mask); lanes holding the same band add
// their counts and differences with one shared atomic per group, edge
// categories are counted per lane in registers and reduced by shuffles.
// k_sao_decide: one warp per CTB, luma, Cb, then Cr within Cb's type
// (src/sao_enc.rs:450-477).
#include <climits>

#include <cstring>

#include "internal.h"

namespace h266 {
namespace {

constexpr int kStatThreads = 256;
constexpr int kSliceRows = 16;

struct SaoStats {  // one (CTB, component)
  long long bo_cnt[32], bo_dif[32];
  long long eo_cnt[4][5], eo_dif[4][5];  // category 0 is not gathered (the decision never reads it)
};

struct SaoEncArgs {
  DPlane src[3], rec[3];
  int bd, log2, w_ctbs, h_ctbs, luma_on, chroma_on;
};

// The CTB region of component c (src/sao_enc.rs:398-420), clipped to the plane
// as try_band_offset / try_edge_offset_class do (x_end, y_end).
__device__ __forceinline__ bool sao_region(const SaoEncArgs &a, int c, int rx, int ry, int &x0, int &y0, int &x1,
                                           int &y1) {
  const int ctb = 1 << a.log2, pw = a.rec[0].w, ph = a.rec[0].h;
  const int cx = rx * ctb, cy = ry * ctb, cw = min(ctb, pw - cx), ch = min(ctb, ph - cy);
  if (c == 0) {
    x0 = cx;
    y0 = cy;
    x1 = min(cx + cw, a.rec[0].w);
    y1 = min(cy + ch, a.rec[0].h);
    return true;
  }
  if (cw / 2 <= 0 || ch / 2 <= 0) return false;
  x0 = cx / 2;
  y0 = cy / 2;
  x1 = min(x0 + cw / 2, a.rec[c].w);
  y1 = min(y0 + ch / 2, a.rec[c].h);
  return true;
}

__device__ __forceinline__ int eo_cat(int r, int n0, int n1) {  // eo_category, src/sao_enc.rs:349-373
  const int s = (r > n0) - (r < n0) + (r > n1) - (r < n1);
  return s == 2 ? 4 : (s == 1 ? 3 : (s == -1 ? 2 : (s == -2 ? 1 : 0)));
}

// Adds (1, d) into bins[key] for every lane with key >= 0, one atomic per
// group of lanes sharing a key.  Called by all 32 lanes.
__device__ __forceinline__ void group_add(int key, int d, unsigned int *cnt, unsigned long long *dif) {
  const unsigned m = __match_any_sync(0xffffffffu, key);
  const int sum = __reduce_add_sync(m, d);
  if (key >= 0 && (int)(threadIdx.x & 31) == __ffs(m) - 1) {
    atomicAdd(cnt + key, (unsigned)__popc(m));
    atomicAdd(dif + key, (unsigned long long)(long long)sum);
  }
}

// Statistics are added into the zeroed `out` with global atomics.
__global__ void __launch_bounds__(kStatThreads) k_sao_stats(const __grid_constant__ SaoEncArgs a,
                                                            SaoStats *__restrict__ out, uint32_t *__restrict__ err) {
  const int ctb_i = blockIdx.x, c = blockIdx.y;
  const int rx = ctb_i % a.w_ctbs, ry = ctb_i / a.w_ctbs;
  int x0, y0, x1, y1;
  if (!(c == 0 ? a.luma_on : a.chroma_on) || !sao_region(a, c, rx, ry, x0, y0, x1, y1)) return;
  y0 += blockIdx.z * kSliceRows;
  y1 = min(y1, y0 + kSliceRows);
  if (x1 <= x0 || y1 <= y0) return;  // uniform per CTA
  __shared__ unsigned int s_bo_cnt[32];
  __shared__ unsigned long long s_bo_dif[32];
  __shared__ int s_eo[2][16];
  const int tid = threadIdx.x, lane = tid & 31;
  if (tid < 32) {
    s_bo_cnt[tid] = 0;
    s_bo_dif[tid] = 0;
    s_eo[0][tid & 15] = 0;
    s_eo[1][tid & 15] = 0;
  }
  __syncthreads();
  const DPlane R = a.rec[c], S = a.src[c];
  const int w = x1 - x0;
  const int shift = a.bd - 5;
  int ecnt[16], edif[16];  // [class * 4 + category - 1]
#pragma unroll
  for (int k = 0; k < 16; ++k) ecnt[k] = edif[k] = 0;
  // a warp per row, 32 columns per step; whole warps step together
  for (int y = y0 + (tid >> 5); y < y1; y += kStatThreads / 32)
    for (int xo = 0; xo < w; xo += 32) {
      const bool in = xo + lane < w;
      const int x = x0 + (in ? xo + lane : 0);
      const int r = (int)R.s[(int64_t)y * R.stride + x];
      const bool sv = in && x < S.w && y < S.h;
      const int d = sv ? (int)S.s[(int64_t)y * S.stride + x] - r : 0;
      int band = sv ? (r >> shift) : -1;
      if (band > 31) {  // a sample above 2^BitDepth - 1: no band in the crate
        atomicOr(err, 1u);
        band = -1;
      }
      group_add(band, d, s_bo_cnt, s_bo_dif);
      if (sv) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {  // EO_DIRS, src/sao_enc.rs:166-171 (second neighbour = -first)
          const int dx0 = k == 1 ? 0 : (k == 3 ? 1 : -1), dy0 = k == 0 ? 0 : -1;
          const int ax = x + dx0, ay = y + dy0, bx = x - dx0, by = y - dy0;
          if (ax >= 0 && ay >= 0 && bx >= 0 && by >= 0 && ax < R.w && ay < R.h && bx < R.w && by < R.h) {
            const int cat = eo_cat(r, R.s[(int64_t)ay * R.stride + ax], R.s[(int64_t)by * R.stride + bx]);
#pragma unroll
            for (int q = 1; q <= 4; ++q) {
              ecnt[k * 4 + q - 1] += cat == q;
              edif[k * 4 + q - 1] += cat == q ? d : 0;
            }
          }
        }
      }
    }
#pragma unroll
  for (int k = 0; k < 16; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ecnt[k] += __shfl_down_sync(0xffffffffu, ecnt[k], o);
      edif[k] += __shfl_down_sync(0xffffffffu, edif[k], o);
    }
  }
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      atomicAdd(&s_eo[0][k], ecnt[k]);
      atomicAdd(&s_eo[1][k], edif[k]);
    }
  __syncthreads();
  SaoStats &o = out[(size_t)ctb_i * 3 + c];
  if (tid < 32) {
    if (s_bo_cnt[tid]) {
      atomicAdd(reinterpret_cast<unsigned long long *>(&o.bo_cnt[tid]), (unsigned long long)s_bo_cnt[tid]);
      atomicAdd(reinterpret_cast<unsigned long long *>(&o.bo_dif[tid]), s_bo_dif[tid]);
    }
  } else if (tid < 48) {
    const int k = tid - 32;
    atomicAdd(reinterpret_cast<unsigned long long *>(&o.eo_cnt[k / 4][k % 4 + 1]),
              (unsigned long long)(long long)s_eo[0][k]);
    atomicAdd(reinterpret_cast<unsigned long long *>(&o.eo_dif[k / 4][k % 4 + 1]),
              (unsigned long long)(long long)s_eo[1][k]);
  }
}

__device__ void sao_offsets(h266_sao_ctb &c, const int abs_[4], const uint32_t sign[4], int bd) {
  const int shift = bd - min(bd, 10);  // derive_offset_val, src/sao.rs:356-365
  c.offset_val[0] = 0;
  for (int i = 0; i < 4; ++i) c.offset_val[i + 1] = (1 - 2 * (int)(sign[i] & 1)) * (abs_[i] << shift);
}

// Band and edge candidates of one component from its statistics, one warp
// (every lane returns the same values):
//  * try_band_offset (src/sao_enc.rs:77-171): lane b holds band b's clipped
//    optimum; lane st < 28 the delta of the 4 bands from st; the first
//    minimum wins (the crate's strict < scan from start 0);
//  * try_edge_offset_class (src/sao_enc.rs:211-284): lane 4k + q - 1 holds
//    category q of class k (offset from |diff|, as there).
struct Candidates {
  long long bo_delta;
  int bo_start, bo_off[4];
  long long eo_delta[4];
  int eo_off[4][4];
};

__device__ Candidates candidates(const SaoStats &s, int bd, int lane) {
  Candidates c;
  const long long cmax = (1ll << (min(bd, 10) - 5)) - 1;
  const long long n = s.bo_cnt[lane], dif = s.bo_dif[lane];
  long long opt = 0;
  if (n > 0) {
    opt = (dif + n / 2) / n;
    opt = opt < -cmax ? -cmax : (opt > cmax ? cmax : opt);
  }
  const long long term = n > 0 ? dif * opt : 0;
  long long delta = -(term + __shfl_down_sync(0xffffffffu, term, 1) + __shfl_down_sync(0xffffffffu, term, 2) +
                      __shfl_down_sync(0xffffffffu, term, 3));
  if (lane >= 28) delta = LLONG_MAX;
  int idx = lane;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const long long ov = __shfl_xor_sync(0xffffffffu, delta, o);
    const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
    if (ov < delta || (ov == delta && oi < idx)) {
      delta = ov;
      idx = oi;
    }
  }
  c.bo_delta = delta;
  c.bo_start = idx;
#pragma unroll
  for (int i = 0; i < 4; ++i) c.bo_off[i] = (int)__shfl_sync(0xffffffffu, opt, idx + i);
  const int k = (lane >> 2) & 3, q = (lane & 3) + 1;
  const long long en = lane < 16 ? s.eo_cnt[k][q] : 0;
  const long long ad = lane < 16 ? (s.eo_dif[k][q] < 0 ? -s.eo_dif[k][q] : s.eo_dif[k][q]) : 0;
  long long eo = 0;
  if (en > 0) {
    eo = (ad + en / 2) / en;
    eo = eo < 0 ? 0 : (eo > 7 ? 7 : eo);
  }
  long long et = ad * eo;
  et += __shfl_xor_sync(0xffffffffu, et, 1);
  et += __shfl_xor_sync(0xffffffffu, et, 2);
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    c.eo_delta[kk] = -__shfl_sync(0xffffffffu, et, 4 * kk);
#pragma unroll
    for (int qq = 0; qq < 4; ++qq) c.eo_off[kk][qq] = (int)__shfl_sync(0xffffffffu, eo, 4 * kk + qq);
  }
  return c;
}

__device__ h266_sao_ctb band_ctb(const Candidates &c, int bd) {  // SaoCtb::band_offset, src/sao.rs:150-167
  h266_sao_ctb out{};
  int ab[4];
  uint32_t sg[4];
  for (int i = 0; i < 4; ++i) {
    ab[i] = c.bo_off[i] < 0 ? -c.bo_off[i] : c.bo_off[i];
    sg[i] = c.bo_off[i] < 0 ? 1u : 0u;
  }
  out.sao_type_idx = 1;
  out.band_position = (uint8_t)(c.bo_start & 31);
  sao_offsets(out, ab, sg, bd);
  return out;
}

__device__ h266_sao_ctb edge_ctb(const Candidates &c, int cls, int bd) {  // SaoCtb::edge_offset, src/sao.rs:169-180
  h266_sao_ctb out{};
  const uint32_t sign[4] = {0, 0, 1, 1};
  out.sao_type_idx = 2;
  out.eo_class = (uint8_t)cls;
  sao_offsets(out, c.eo_off[cls], sign, bd);
  return out;
}

__device__ h266_sao_ctb decide(const Candidates &c, int bd) {  // sao_decide_ctb, src/sao_enc.rs:44-70
  long long best = 0;
  int cls = -1;
  for (int k = 0; k < 4; ++k)  // try_best_edge_offset, src/sao_enc.rs:175-209
    if (c.eo_delta[k] < best) {
      best = c.eo_delta[k];
      cls = k;
    }
  if (cls >= 0) return edge_ctb(c, cls, bd);
  if (c.bo_delta < 0) return band_ctb(c, bd);
  return h266_sao_ctb{};
}

// One warp per CTB.
__global__ void k_sao_decide(const __grid_constant__ SaoEncArgs a, const SaoStats *__restrict__ st,
                             h266_sao_ctb_params *__restrict__ out) {
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (i >= a.w_ctbs * a.h_ctbs) return;  // uniform per warp
  const int rx = i % a.w_ctbs, ry = i / a.w_ctbs;
  h266_sao_ctb_params p{};
  if (a.luma_on) {
    const Candidates c = candidates(st[(size_t)i * 3], a.bd, lane);
    p.luma = decide(c, a.bd);
  }
  int x0, y0, x1, y1;
  if (a.chroma_on && sao_region(a, 1, rx, ry, x0, y0, x1, y1)) {
    const Candidates cb = candidates(st[(size_t)i * 3 + 1], a.bd, lane);
    const Candidates cr = candidates(st[(size_t)i * 3 + 2], a.bd, lane);
    p.cb = decide(cb, a.bd);
    if (p.cb.sao_type_idx == 1) {  // sao_decide_ctb_constrained, src/sao_enc.rs:286-347
      if (cr.bo_delta < 0) {
        p.cr = band_ctb(cr, a.bd);
      } else {
        p.cr.sao_type_idx = 1;
      }
    } else if (p.cb.sao_type_idx == 2) {
      const int cls = p.cb.eo_class;
      if (cr.eo_delta[cls] < 0) {
        p.cr = edge_ctb(cr, cls, a.bd);
      } else {
        p.cr.sao_type_idx = 2;
        p.cr.eo_class = (uint8_t)cls;
      }
    }
  }
  if (lane == 0) out[i] = p;
}

// ---- chroma SAO merge (apply_chroma_sao_merge, src/sao_enc.rs:500-668)
//
// Raster-order dependency: a CTB weighs its own parameters against the
// already merged left and above CTBs, so CTBs run one anti-diagonal per
// launch (both neighbours lie on the previous diagonal).  Per CTB and
// candidate: the SAO of this CTB alone on the pre-SAO planes
// (apply_sao_ctb, src/sao.rs:504-626, no clip rectangle) and the Cb + Cr SSE
// against the original (chroma_ctb_sse_with, src/sao_enc.rs:698-749), then
// the decision by cost SSE + 8 * bits (strict <: independent, left, above).
struct MergeArgs {
  DPlane src[2], pre[2];  // Cb, Cr
  int bd, chr_ctb, w_ctbs, diag, first_ry;
  const h266_sao_ctb_params *indep;
  h266_sao_ctb_params *merged;
  uint8_t *map;
  unsigned long long *sse;  // [ctb][3]
  unsigned int *count;      // per CTB, zero at the start
};

__device__ __forceinline__ int sao_value(const DPlane &P, int x, int y, const h266_sao_ctb &p, int maxv, int bd) {
  const int v = P.s[(int64_t)y * P.stride + x];
  if (p.sao_type_idx == 2) {
    const int c = p.eo_class & 3;
    const int hx = c == 1 ? 0 : (c == 3 ? 1 : -1), vy = c == 0 ? 0 : -1;  // hPos / vPos of neighbour 0
    const int ax = x + hx, ay = y + vy, bx = x - hx, by = y - vy;
    if (ax < 0 || ay < 0 || bx < 0 || by < 0 || ax >= P.w || ay >= P.h || bx >= P.w || by >= P.h)
      return min(max(v, 0), maxv);
    const int n0 = P.s[(int64_t)ay * P.stride + ax], n1 = P.s[(int64_t)by * P.stride + bx];
    int e = 2 + ((v > n0) - (v < n0)) + ((v > n1) - (v < n1));
    if (e <= 2) e = e == 2 ? 0 : e + 1;
    const int off = (e >= 1 && e <= 4) ? p.offset_val[e] : 0;
    return min(max(v + off, 0), maxv);
  }
  if (p.sao_type_idx == 1) {
    const int band = (v >> (bd - 5)) & 31;
    const int k = (band - p.band_position) & 31;
    const int off = k < 4 ? p.offset_val[k + 1] : 0;
    return min(max(v + off, 0), maxv);
  }
  return v;  // not applied: the sample as it is
}

constexpr int kMergeThreads = 512;

// One CTA per (CTB of the diagonal, candidate): the candidate's Cb + Cr SSE,
// stored per CTB; the CTA that completes a CTB's set of candidates (per-CTB
// arrival counter, zeroed by the host; no CTA waits for another) makes the
// decision.
__device__ __forceinline__ void merge_cta(const MergeArgs &a, int ry, int rx, int k) {
  if ((k == 1 && rx == 0) || (k == 2 && ry == 0)) return;  // no such neighbour (uniform per CTA)
  const int i = ry * a.w_ctbs + rx;
  const int tid = threadIdx.x, maxv = (1 << a.bd) - 1;
  const int cx = rx * a.chr_ctb, cy = ry * a.chr_ctb;
  const int cw = max(0, min(a.chr_ctb, a.pre[0].w - cx)), ch = max(0, min(a.chr_ctb, a.pre[0].h - cy));
  const h266_sao_ctb_params &cand = k == 0 ? a.indep[i] : (k == 1 ? a.merged[i - 1] : a.merged[i - a.w_ctbs]);
  const h266_sao_ctb pc[2] = {cand.cb, cand.cr};
  unsigned long long e = 0;
  for (int y = cy + tid / 32; y < cy + ch; y += kMergeThreads / 32)
    for (int x = cx + (tid & 31); x < cx + cw; x += 32)
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int d = (int)a.src[c].s[(int64_t)y * a.src[c].stride + x] - sao_value(a.pre[c], x, y, pc[c], maxv, a.bd);
        e += (unsigned long long)((long long)d * d);
      }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
  __shared__ unsigned long long part[kMergeThreads / 32];
  if ((tid & 31) == 0) part[tid / 32] = e;
  __syncthreads();
  if (tid) return;
  unsigned long long t = 0;
  for (int w = 0; w < kMergeThreads / 32; ++w) t += part[w];
  a.sse[(size_t)i * 3 + k] = t;
  __threadfence();
  const unsigned n_cand = 1u + (rx > 0) + (ry > 0);
  if (atomicAdd(&a.count[i], 1u) != n_cand - 1) return;
  __threadfence();
  unsigned long long sse[3];
  for (int q = 0; q < 3; ++q) sse[q] = __ldcg(&a.sse[(size_t)i * 3 + q]);
  auto bits = [](const h266_sao_ctb_params &p) {  // chroma_independent_bit_cost, src/sao_enc.rs:670-696
    long long b = 1;
    b += p.cb.sao_type_idx == 0 ? 1 : (p.cb.sao_type_idx == 1 ? 16 : 10);
    b += p.cr.sao_type_idx == 0 ? 1 : (p.cr.sao_type_idx == 1 ? 16 : 10);
    return b;
  };
  const h266_sao_ctb_params in = a.indep[i];
  long long best = (long long)sse[0] + 8 * bits(in);
  int choice = 0;
  h266_sao_ctb_params out = in;
  if (rx > 0 && (long long)sse[1] + 8 < best) {
    best = (long long)sse[1] + 8;
    choice = 1;
    out.cb = a.merged[i - 1].cb;
    out.cr = a.merged[i - 1].cr;
  }
  if (ry > 0 && (long long)sse[2] + 16 < best) {
    choice = 2;
    out.cb = a.merged[i - a.w_ctbs].cb;
    out.cr = a.merged[i - a.w_ctbs].cr;
  }
  a.merged[i] = out;
  a.map[i] = (uint8_t)choice;
}

__global__ void __launch_bounds__(kMergeThreads) k_sao_merge_diag(const __grid_constant__ MergeArgs a) {
  const int ry = a.first_ry + blockIdx.x;
  merge_cta(a, ry, a.diag - ry, blockIdx.y);
}

// One anti-diagonal `diag` of many pictures: CTAs [first[p], first[p + 1]) of
// the x dimension are picture p's CTBs on it (from its first row up), y the
// candidate.  Pictures without CTBs on the diagonal have none.
__global__ void __launch_bounds__(kMergeThreads) k_sao_merge_diag_batch(const MergeArgs *__restrict__ args,
                                                                         const uint32_t *__restrict__ first, int n,
                                                                         int diag) {
  int lo = 0, hi = n;  // first[lo] <= blockIdx.x < first[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (first[mid] <= blockIdx.x) lo = mid;
    else hi = mid;
  }
  const MergeArgs &a = args[lo];
  const int ry0 = max(0, diag - (a.w_ctbs - 1));
  const int ry = ry0 + (int)(blockIdx.x - first[lo]);
  merge_cta(a, ry, diag - ry, blockIdx.y);
}

}  // namespace

size_t sao_merge_args_size() { return sizeof(MergeArgs); }

void fill_sao_merge_args(void *out, const DPlane src[2], const DPlane pre[2], int bd, int chr_ctb, int w_ctbs,
                         int h_ctbs, const h266_sao_ctb_params *d_indep, h266_sao_ctb_params *d_merged, uint8_t *d_map,
                         void *d_work) {
  MergeArgs a{};
  for (int c = 0; c < 2; ++c) {
    a.src[c] = src[c];
    a.pre[c] = pre[c];
  }
  a.bd = bd;
  a.chr_ctb = chr_ctb;
  a.w_ctbs = w_ctbs;
  a.indep = d_indep;
  a.merged = d_merged;
  a.map = d_map;
  a.sse = static_cast<unsigned long long *>(d_work);  // the layout of sao_merge_work_bytes; counts zeroed by the caller
  a.count = reinterpret_cast<unsigned int *>(a.sse + (size_t)w_ctbs * h_ctbs * 3);
  std::memcpy(out, &a, sizeof a);
}

int launch_sao_chroma_merge_batch(cudaStream_t st, const void *d_args, const uint32_t *d_first, int n, int n_diags,
                                  const uint32_t *h_totals, uint64_t *launches) {
  const MergeArgs *args = static_cast<const MergeArgs *>(d_args);
  for (int d = 0; d < n_diags; ++d) {
    if (!h_totals[d]) continue;
    k_sao_merge_diag_batch<<<dim3(h_totals[d], 3), kMergeThreads, 0, st>>>(args, d_first + (size_t)d * (n + 1), n, d);
    H266_CUDA(cudaGetLastError());
    ++*launches;
  }
  return H266_OK;
}

int launch_sao_chroma_merge(cudaStream_t st, const DPlane src[2], const DPlane pre[2], int bd, int chr_ctb,
                            int w_ctbs, int h_ctbs, const h266_sao_ctb_params *d_indep, h266_sao_ctb_params *d_merged,
                            uint8_t *d_map, void *d_work, uint64_t *launches) {
  MergeArgs a{};
  a.sse = static_cast<unsigned long long *>(d_work);
  a.count = reinterpret_cast<unsigned int *>(a.sse + (size_t)w_ctbs * h_ctbs * 3);
  H266_CUDA(cudaMemsetAsync(a.count, 0, (size_t)w_ctbs * h_ctbs * sizeof(unsigned int), st));
  for (int c = 0; c < 2; ++c) {
    a.src[c] = src[c];
    a.pre[c] = pre[c];
  }
  a.bd = bd;
  a.chr_ctb = chr_ctb;
  a.w_ctbs = w_ctbs;
  a.indep = d_indep;
  a.merged = d_merged;
  a.map = d_map;
  for (int d = 0; d <= w_ctbs + h_ctbs - 2; ++d) {
    const int ry0 = max(0, d - (w_ctbs - 1)), ry1 = min(h_ctbs - 1, d);
    a.diag = d;
    a.first_ry = ry0;
    k_sao_merge_diag<<<dim3(ry1 - ry0 + 1, 3), kMergeThreads, 0, st>>>(a);
    H266_CUDA(cudaGetLastError());
    ++*launches;
  }
  return H266_OK;
}

size_t sao_stats_bytes(int n_ctbs) { return (size_t)n_ctbs * 3 * sizeof(SaoStats); }

int launch_sao_decide(cudaStream_t st, const DPlane src[3], const DPlane rec[3], int bd, int log2, int w_ctbs,
                      int h_ctbs, bool luma_on, bool chroma_on, void *d_stats, uint32_t *d_err,
                      h266_sao_ctb_params *d_out, uint64_t *launches) {
  const int n = w_ctbs * h_ctbs;
  if (n <= 0) return H266_OK;
  SaoEncArgs a{};
  for (int i = 0; i < 3; ++i) {
    a.src[i] = src[i];
    a.rec[i] = rec[i];
  }
  a.bd = bd;
  a.log2 = log2;
  a.w_ctbs = w_ctbs;
  a.h_ctbs = h_ctbs;
  a.luma_on = luma_on;
  a.chroma_on = chroma_on;
  auto *stats = static_cast<SaoStats *>(d_stats);
  H266_CUDA(cudaMemsetAsync(stats, 0, sao_stats_bytes(n), st));
  const int slices = ((1 << log2) + kSliceRows - 1) / kSliceRows;
  k_sao_stats<<<dim3(n, 3, slices), kStatThreads, 0, st>>>(a, stats, d_err);
  H266_CUDA(cudaGetLastError());
  k_sao_decide<<<(n * 32 + 127) / 128, 128, 0, st>>>(a, stats, d_out);
  H266_CUDA(cudaGetLastError());
  *launches += 2;
  return H266_OK;
}

}  // namespace h266
