// LMCS for the filter chain: the §7.4.3.19 derivation (host) and the §8.8.2
// inverse luma map as a 65536-entry device LUT applied while copying a plane.
#include "internal.h"

namespace h266 {

// derive_lmcs, src/lmcs.rs:302-404 (every conformance clause of §7.4.3.19).
int derive_lmcs(const h266_lmcs_data *d, uint32_t bd, h266_lmcs_derived *o) {
  if (!d || !o) return set_error(H266_ERR_INVALID_ARGUMENT, "derive_lmcs: NULL argument");
  *o = h266_lmcs_derived{};
  if (bd < 8 || bd > 16) return set_error(H266_ERR_LMCS_CONFORMANCE, "LMCS: BitDepth out of range 8..16");
  if (d->lmcs_delta_max_bin_idx > 15 || d->lmcs_min_bin_idx > 15)
    return set_error(H266_ERR_LMCS_CONFORMANCE, "LMCS: bin index out of range");
  const uint32_t org = (1u << bd) / 16, log2org = bd - 4;
  const int64_t lo = org >> 3, hi = (int64_t)(org << 3) - 1;
  const uint32_t mn = d->lmcs_min_bin_idx, mx = 15u - d->lmcs_delta_max_bin_idx;
  uint32_t cw[16] = {0};
  for (uint32_t i = mn; i <= mx; ++i) {
    const int64_t v = (int64_t)org + (d->lmcs_delta_sign_cw_flag[i] ? -1 : 1) * (int64_t)d->lmcs_delta_abs_cw[i];
    if (v < lo || v > hi) return set_error(H266_ERR_LMCS_CONFORMANCE, "LMCS: lmcsCW outside the eq. 95 band");
    cw[i] = (uint32_t)v;
  }
  uint64_t total = 0;
  for (uint32_t c : cw) total += c;
  if (total > (1u << bd) - 1) return set_error(H266_ERR_LMCS_CONFORMANCE, "LMCS: sum of lmcsCW exceeds the budget");
  o->lmcs_pivot[0] = 0;
  for (uint32_t i = 0; i < 16; ++i) {
    o->lmcs_cw[i] = cw[i];
    o->input_pivot[i] = i * org;
    o->lmcs_pivot[i + 1] = o->lmcs_pivot[i] + cw[i];
    o->scale_coeff[i] = (cw[i] * 2048u + (1u << (log2org - 1))) >> log2org;
    o->inv_scale_coeff[i] = cw[i] ? org * 2048u / cw[i] : 0;
  }
  const uint32_t sh = bd - 5;
  for (uint32_t i = mn; i <= mx; ++i)
    if (o->lmcs_pivot[i] % (1u << sh) != 0 && (o->lmcs_pivot[i] >> sh) == (o->lmcs_pivot[i + 1] >> sh))
      return set_error(H266_ERR_LMCS_CONFORMANCE, "LMCS: LmcsPivot bin-crossing clause violated");
  const int32_t crs = (d->lmcs_delta_sign_crs_flag ? -1 : 1) * (int32_t)d->lmcs_delta_abs_crs;
  for (uint32_t i = 0; i < 16; ++i) {
    if (cw[i] == 0) {
      o->chroma_scale_coeff[i] = 2048;
      continue;
    }
    const int64_t j = (int64_t)cw[i] + crs;
    if (j < lo || j > hi) return set_error(H266_ERR_LMCS_CONFORMANCE, "LMCS: lmcsCW + lmcsDeltaCrs outside the band");
    o->chroma_scale_coeff[i] = org * 2048u / (uint32_t)j;
  }
  o->bit_depth = bd;
  o->org_cw = org;
  o->lmcs_delta_crs = crs;
  return H266_OK;
}

namespace {

struct LmcsTables {
  uint32_t pivot[17];
  uint32_t input_pivot[16];
  uint32_t inv_scale[16];
  uint32_t mn, mx, maxv;
};

// One LUT entry per u16 input: idx_y_inv then inverse_map_luma_sample
// (src/lmcs.rs:209-238), exactly the per-sample fold of src/ctu.rs:11841-11848.
__global__ void k_lmcs_lut(uint16_t *lut, LmcsTables t) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= 65536) return;
  uint32_t idx = t.mn;
  while (idx <= t.mx && s >= t.pivot[idx + 1]) ++idx;
  idx = min(idx, 15u);
  const int64_t prod = (int64_t)t.inv_scale[idx] * ((int64_t)s - (int64_t)t.pivot[idx]) + 1024;
  const int64_t inv = (int64_t)t.input_pivot[idx] + (prod >> 11);
  lut[s] = (uint16_t)(inv < 0 ? 0 : (inv > (int64_t)t.maxv ? t.maxv : inv));
}

// dst = lut ? lut[src] : src, 8 samples per thread along a row.
__global__ void k_plane_map(DPlane dst, DPlane src, const uint16_t *__restrict__ lut) {
  const int y = blockIdx.y;
  const int x0 = (blockIdx.x * blockDim.x + threadIdx.x) * 8;
  if (y >= src.h || x0 >= src.w) return;
  const uint16_t *s = src.s + (int64_t)y * src.stride;
  uint16_t *d = dst.s + (int64_t)y * dst.stride;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int x = x0 + i;
    if (x < src.w) {
      const uint16_t v = s[x];
      d[x] = lut ? lut[v] : v;
    }
  }
}

}  // namespace

int launch_lmcs_lut(cudaStream_t st, uint16_t *d_lut, const h266_lmcs_derived &l, uint32_t mn, uint32_t mx,
                    uint64_t *launches) {
  if (l.bit_depth < 8 || l.bit_depth > 16) return set_error(H266_ERR_INVALID_ARGUMENT, "LMCS: bad bit_depth");
  if (mn > 15 || mx > 15) return set_error(H266_ERR_INVALID_ARGUMENT, "LMCS: bin index out of range");
  LmcsTables t;
  for (int i = 0; i < 17; ++i) t.pivot[i] = l.lmcs_pivot[i];
  for (int i = 0; i < 16; ++i) {
    t.input_pivot[i] = l.input_pivot[i];
    t.inv_scale[i] = l.inv_scale_coeff[i];
  }
  t.mn = mn;
  t.mx = mx;
  t.maxv = (1u << l.bit_depth) - 1;
  k_lmcs_lut<<<256, 256, 0, st>>>(d_lut, t);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

int launch_plane_map(cudaStream_t st, DPlane dst, DPlane src, const uint16_t *d_lut, uint64_t *launches) {
  if (src.w <= 0 || src.h <= 0) return H266_OK;
  const int threads = 128;
  dim3 grid((src.w + threads * 8 - 1) / (threads * 8), src.h);
  k_plane_map<<<grid, threads, 0, st>>>(dst, src, d_lut);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

}  // namespace h266
