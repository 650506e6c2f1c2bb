// The steps either side of the filter chain that share its sample layout:
// the recon-side LMCS (forward luma map of inter CUs, chroma residual
// scaling factor and residual add, src/lmcs.rs:169-290, src/ctu.rs:734-742,
// 1701-1815) and the cropped planar output dump (examples/decode_dump.rs).
// All of it is byte / integer work bound by memory latency or bandwidth: one
// CTA per rectangle piece or transform block, a warp per scaling factor, a
// flat grid for the dump.
#include "internal.h"

namespace h266 {
namespace {

constexpr int kPieceThreads = 256;

// Forward LUT, one entry per u16 input (src/lmcs.rs:186-194 then the Clip1 of
// src/ctu.rs:1722): entries above 2^BitDepth - 1 have no bin in the crate and
// hold kNoBin (never a mapped value when BitDepth < 16).
constexpr uint16_t kNoBin = 0xFFFF;
struct FwdTables {
  uint32_t lmcs_pivot[16], input_pivot[16], scale[16];
  uint32_t bd;
};

__global__ void k_lmcs_fwd_lut(uint16_t *lut, FwdTables t) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= 65536) return;
  const uint32_t idx = s >> (t.bd - 4);
  if (idx > 15) {
    lut[s] = kNoBin;
    return;
  }
  const int64_t prod = (int64_t)t.scale[idx] * ((int64_t)s - (int64_t)t.input_pivot[idx]) + 1024;
  const int64_t m = (int64_t)t.lmcs_pivot[idx] + (prod >> 11);
  const int64_t hi = ((int64_t)1 << t.bd) - 1;
  lut[s] = (uint16_t)(m < 0 ? 0 : (m > hi ? hi : m));
}

// One CTA per rectangle piece (<= 4096 samples); pieces of one launch never
// overlap.  A sample without a bin stays as it is and raises *err.
__global__ void __launch_bounds__(kPieceThreads) k_lmcs_fwd_rects(DPlane p, const uint16_t *__restrict__ lut,
                                                                  const RectPiece *__restrict__ pieces, int check,
                                                                  uint32_t *__restrict__ err) {
  const RectPiece r = pieces[blockIdx.x];
  const int n = (int)(r.w * r.h);
  for (int i = threadIdx.x; i < n; i += kPieceThreads) {
    const int y = (int)r.y + i / (int)r.w, x = (int)r.x + i % (int)r.w;
    uint16_t &s = p.s[(int64_t)y * p.stride + x];
    const uint16_t m = __ldg(lut + s);
    if (check && m == kNoBin) {
      atomicOr(err, 1u);
      continue;
    }
    s = m;
  }
}

// One warp per CU (src/ctu.rs:1779-1814).
__global__ void k_lmcs_cvs(DPlane luma, const h266_lmcs_cvs_block *__restrict__ b, int n, int size_y, int log2_cnt1,
                           CvsTables t, uint32_t *__restrict__ out) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n) return;
  const h266_lmcs_cvs_block c = b[w];
  const bool al = c.x_cu_cb > 0 && c.avail_l, at = c.y_cu_cb > 0 && c.avail_t;
  uint32_t sum = 0;
  for (int i = lane; i < size_y; i += 32) {
    if (al) {
      const int yy = min((int)c.y_cu_cb + i, luma.h - 1);
      sum += luma.s[(int64_t)yy * luma.stride + (c.x_cu_cb - 1)];
    }
    if (at) {
      const int xx = min((int)c.x_cu_cb + i, luma.w - 1);
      sum += luma.s[(int64_t)(c.y_cu_cb - 1) * luma.stride + xx];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
  if (lane) return;
  const int sides = (al ? 1 : 0) + (at ? 1 : 0);
  uint32_t avg;
  if (sides) {
    const int sh = log2_cnt1 + (sides == 2 ? 1 : 0);  // Log2(cnt), cnt = sizeY or 2 sizeY
    avg = (uint32_t)(((uint64_t)sum + ((uint64_t)1 << sh >> 1)) >> sh);
  } else {
    avg = 1u << (t.bd - 1);
  }
  uint32_t idx = t.mn;  // idx_y_inv, src/lmcs.rs:209-221
  while (idx <= t.mx && avg >= t.pivot[idx + 1]) ++idx;
  out[w] = t.chroma_scale[min(idx, 15u)];
}

// One CTA per chroma TB (<= 4096 samples after the host's row split); TBs of
// one launch never overlap.
__global__ void __launch_bounds__(kPieceThreads) k_chroma_residual(DPlane cb, DPlane cr,
                                                                   const ResPiece *__restrict__ pieces,
                                                                   const int32_t *__restrict__ res, int bd) {
  const ResPiece r = pieces[blockIdx.x];
  const DPlane &p = r.plane == 1 ? cb : cr;
  const int n = (int)(r.w * r.h);
  const int64_t lo = -((int64_t)1 << bd), hi = ((int64_t)1 << bd) - 1;
  for (int i = threadIdx.x; i < n; i += kPieceThreads) {
    const int row = i / (int)r.w, col = i % (int)r.w;
    int64_t v = res[r.res_offset + (uint64_t)row * r.res_pitch + col];
    if (r.var_scale != H266_NO_VAR_SCALE) {  // eqs. 1219 / 1220
      v = v < lo ? lo : (v > hi ? hi : v);
      const int64_t mag = (int64_t)(((uint64_t)(v < 0 ? -v : v) * r.var_scale + 1024) >> 11);
      v = v < 0 ? -mag : mag;
    }
    uint16_t &s = p.s[(int64_t)(r.y + row) * p.stride + r.x + col];
    const int64_t o = (int64_t)s + v;
    s = (uint16_t)(o < 0 ? 0 : (o > hi ? hi : o));
  }
}

// The dump: one thread per 4 output samples of the flattened luma / Cb / Cr
// crops; 8-bit output is the low byte of each sample, wider output the
// little-endian u16 (the device is little-endian, so a u16 store).
__global__ void k_output_dump(OutPlanes o, uint8_t *__restrict__ dst, int wide) {
  const uint64_t q = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint64_t i = q + k;
    if (i >= o.total) return;
    int pl = 0;
    uint64_t j = i;
    if (j >= o.n[0]) {
      j -= o.n[0];
      pl = 1;
      if (j >= o.n[1]) {
        j -= o.n[1];
        pl = 2;
      }
    }
    const uint32_t w = o.w[pl];
    const uint32_t y = (uint32_t)(j / w), x = (uint32_t)(j - (uint64_t)y * w);
    const uint16_t v = o.p[pl].s[(int64_t)(o.y0[pl] + y) * o.p[pl].stride + o.x0[pl] + x];
    if (wide) reinterpret_cast<uint16_t *>(dst)[i] = v;
    else dst[i] = (uint8_t)v;
  }
}

}  // namespace

int launch_lmcs_fwd_lut(cudaStream_t st, uint16_t *d_lut, const h266_lmcs_derived &l, uint64_t *launches) {
  FwdTables t;
  for (int i = 0; i < 16; ++i) {
    t.lmcs_pivot[i] = l.lmcs_pivot[i];
    t.input_pivot[i] = l.input_pivot[i];
    t.scale[i] = l.scale_coeff[i];
  }
  t.bd = l.bit_depth;
  k_lmcs_fwd_lut<<<256, 256, 0, st>>>(d_lut, t);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

int launch_lmcs_fwd_rects(cudaStream_t st, DPlane p, const uint16_t *d_lut, const RectPiece *d_pieces, uint32_t n,
                          bool check, uint32_t *d_err, uint64_t *launches) {
  if (!n) return H266_OK;
  k_lmcs_fwd_rects<<<n, kPieceThreads, 0, st>>>(p, d_lut, d_pieces, check ? 1 : 0, d_err);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

int launch_lmcs_cvs(cudaStream_t st, DPlane luma, const h266_lmcs_cvs_block *d_blocks, uint32_t n, int size_y,
                    const CvsTables &t, uint32_t *d_out, uint64_t *launches) {
  if (!n) return H266_OK;
  int l = 0;
  while ((1 << l) < size_y) ++l;
  const uint64_t threads = (uint64_t)n * 32;
  k_lmcs_cvs<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(luma, d_blocks, (int)n, size_y, l, t, d_out);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

int launch_chroma_residual(cudaStream_t st, DPlane cb, DPlane cr, const ResPiece *d_pieces, uint32_t n,
                           const int32_t *d_res, int bd, uint64_t *launches) {
  if (!n) return H266_OK;
  k_chroma_residual<<<n, kPieceThreads, 0, st>>>(cb, cr, d_pieces, d_res, bd);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

int launch_output_dump(cudaStream_t st, const OutPlanes &o, uint8_t *d_dst, bool wide, uint64_t *launches) {
  if (!o.total) return H266_OK;
  const uint64_t threads = (o.total + 3) / 4;
  k_output_dump<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(o, d_dst, wide ? 1 : 0);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

}  // namespace h266
