// The steps either side of the filter chain that share its sample layout:
// the recon-side LMCS (forward luma map of inter CUs, chroma residual
// scaling factor and residual add, src/lmcs.rs:169-290, src/ctu.rs:734-742,
// 1701-1815) and the cropped planar output dump (examples/decode_dump.rs).
// All of it is byte / integer work bound by memory latency or bandwidth: a
// coverage count and one pass over the rectangles' span for the forward map,
// a warp per transform-block piece, a warp per scaling factor, a flat grid
// for the dump.
#include "internal.h"

namespace h266 {
namespace {

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

// Coverage count: one warp per rectangle piece, one counter increment per
// grid cell of the piece (pieces hold at most 1024 cells and lie on the grid).
__global__ void k_lmcs_fwd_count(const RectPiece *__restrict__ pieces, uint32_t n, FwdCover c) {
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n) return;
  const RectPiece r = pieces[w];
  const uint32_t cx = r.x >> c.sh, cy = r.y >> c.sh, nw = r.w >> c.sh, nh = r.h >> c.sh;
  for (uint32_t i = lane; i < nw * nh; i += 32) atomicAdd(&c.cnt[(size_t)(cy + i / nw) * c.pitch + cx + i % nw], 1u);
}

// The map itself over the span box: 8 samples of a row per thread (one
// 16-byte load and store where the plane allows), each mapped as many times
// as rectangles cover its cell, so a sample inside k rectangles gets the
// crate's k successive maps (the same table each time, so the rectangles'
// order does not change the result).  A sample without a bin stays as it is
// and raises *err; the mapped value of a sample with a bin always has one.
// A CTA covers 256 columns and 8 rows, whole grid cells (the grid is at most
// 4 samples and the box starts on it), so after its barrier it sets the
// counters it read back to zero: the counter array stays zeroed between calls.
constexpr int kBoxRows = 8;
__global__ void __launch_bounds__(256) k_lmcs_fwd_apply(DPlane p, const uint16_t *__restrict__ lut, FwdCover c,
                                                        int check, int vec, uint32_t *__restrict__ err) {
  const uint32_t y = c.y0 + blockIdx.y * kBoxRows + threadIdx.y;
  const uint32_t x = (c.x0 & ~7u) + (blockIdx.x * 32 + threadIdx.x) * 8;
  const bool live = y < c.y1 && x < c.x1;
  uint32_t *crow = c.cnt + (size_t)(y >> c.sh) * c.pitch;
  if (live) {
    uint32_t k[8], any = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint32_t xx = x + j;
      k[j] = xx >= c.x0 && xx < c.x1 ? crow[xx >> c.sh] : 0;
      any |= k[j];
    }
    if (any) {
      uint16_t *s = p.s + (int64_t)y * p.stride + x;
      auto map = [&](uint16_t v, uint32_t times) {
        for (uint32_t i = 0; i < times; ++i) {
          const uint16_t m = __ldg(lut + v);
          if (check && m == kNoBin) {
            atomicOr(err, 1u);
            break;
          }
          v = m;
        }
        return v;
      };
      if (vec && x + 8 <= (uint32_t)p.w) {
        const uint4 q = *reinterpret_cast<const uint4 *>(s);
        uint32_t wd[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const uint16_t lo = map((uint16_t)(wd[j] & 0xFFFF), k[2 * j]);
          const uint16_t hi = map((uint16_t)(wd[j] >> 16), k[2 * j + 1]);
          wd[j] = (uint32_t)lo | ((uint32_t)hi << 16);
        }
        *reinterpret_cast<uint4 *>(s) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (k[j]) s[j] = map(s[j], k[j]);
      }
    }
  }
  __syncthreads();
  if (live && ((y - c.y0) & ((1u << c.sh) - 1)) == 0) {  // the top row of each grid row clears it
    const uint32_t lo = max(x, c.x0) >> c.sh, hi = (min(x + 8, c.x1) - 1) >> c.sh;
    for (uint32_t cx = lo; cx <= hi; ++cx)
      if (crow[cx]) crow[cx] = 0;
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

// One residual folded by lmcs_scale_chroma_residuals when the TB has a
// varScale (eqs. 1219 / 1220) and added to the sample with Clip1
// (src/ctu.rs:9912-9945); lo / hi: -(1 << bd) and (1 << bd) - 1.
__device__ __forceinline__ uint16_t res_add(uint16_t s, int64_t v, uint32_t var_scale, int64_t lo, int64_t hi) {
  if (var_scale != H266_NO_VAR_SCALE) {
    v = v < lo ? lo : (v > hi ? hi : v);
    const int64_t mag = (int64_t)(((uint64_t)(v < 0 ? -v : v) * var_scale + 1024) >> 11);
    v = v < 0 ? -mag : mag;
  }
  const int64_t o = (int64_t)s + v;
  return (uint16_t)(o < 0 ? 0 : (o > hi ? hi : o));
}

// Ordered form: one warp per chroma TB piece (<= 1024 samples after the
// host's row split), 8 warps per CTA; TBs of one launch never overlap.
constexpr int kResWarps = 8;
__global__ void __launch_bounds__(kResWarps * 32) k_chroma_residual(DPlane cb, DPlane cr,
                                                                   const ResPiece *__restrict__ pieces, uint32_t n_pieces,
                                                                   const int32_t *__restrict__ res, int bd) {
  const uint32_t w = blockIdx.x * kResWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (w >= n_pieces) return;
  const ResPiece r = pieces[w];
  const DPlane &p = r.plane == 1 ? cb : cr;
  const int n = (int)(r.w * r.h);
  const int64_t lo = -((int64_t)1 << bd), hi = ((int64_t)1 << bd) - 1;
  for (int i = lane; i < n; i += 32) {
    const int row = i / (int)r.w, col = i % (int)r.w;
    uint16_t &s = p.s[(int64_t)(r.y + row) * p.stride + r.x + col];
    s = res_add(s, res[r.res_offset + (uint64_t)row * r.res_pitch + col], r.var_scale, lo, hi);
  }
}

// Cell owners: one warp per TB.
__global__ void k_res_own(const h266_chroma_res_block *__restrict__ b, uint32_t n, ResCover c,
                          uint32_t *__restrict__ overlap) {
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n) return;
  const h266_chroma_res_block t = b[w];
  const bool cr = t.plane == 2;
  const uint32_t nw = t.w >> c.sh, nh = t.h >> c.sh, pitch = cr ? c.pitch[1] : c.pitch[0];
  uint32_t *own = (cr ? c.own[1] : c.own[0]) + (size_t)(t.y >> c.sh) * pitch + (t.x >> c.sh);
  uint32_t hit = 0;
  for (uint32_t i = lane; i < nw * nh; i += 32) hit |= atomicCAS(own + (size_t)(i / nw) * pitch + i % nw, 0u, w + 1);
  if (__any_sync(0xFFFFFFFFu, hit != 0) && lane == 0) atomicOr(overlap, 1u);
}

// The add over each plane's box (blockIdx.z: Cb, Cr), 8 samples of a row per
// thread, every sample through its cell's owner TB; a CTA covers 256 columns
// and 8 rows, whole grid cells, and sets the owners it read back to 0 after
// its barrier.
__global__ void __launch_bounds__(256) k_res_apply(DPlane cb, DPlane cr, const h266_chroma_res_block *__restrict__ b,
                                                   const int32_t *__restrict__ res, ResCover c, int bd, int vec,
                                                   const uint32_t *__restrict__ overlap) {
  if (*overlap) return;  // the whole grid returns: the ordered launches follow
  const bool pl = blockIdx.z != 0;
  const DPlane &p = pl ? cr : cb;
  const uint32_t x0 = pl ? c.x0[1] : c.x0[0], x1 = pl ? c.x1[1] : c.x1[0], y0 = pl ? c.y0[1] : c.y0[0];
  const uint32_t y = y0 + blockIdx.y * kBoxRows + threadIdx.y;
  const uint32_t x = (x0 & ~7u) + (blockIdx.x * 32 + threadIdx.x) * 8;
  const bool live = y < (pl ? c.y1[1] : c.y1[0]) && x < x1;
  uint32_t *orow = (pl ? c.own[1] : c.own[0]) + (size_t)(y >> c.sh) * (pl ? c.pitch[1] : c.pitch[0]);
  if (live) {
    const int64_t lo = -((int64_t)1 << bd), hi = ((int64_t)1 << bd) - 1;
    uint16_t *s = p.s + (int64_t)y * p.stride + x;
    const bool v16 = vec && x + 8 <= (uint32_t)p.w;
    uint16_t v[8];
    if (v16) {
      const uint4 q = *reinterpret_cast<const uint4 *>(s);
      const uint32_t wd[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        v[2 * j] = (uint16_t)(wd[j] & 0xFFFF);
        v[2 * j + 1] = (uint16_t)(wd[j] >> 16);
      }
    }
    uint32_t last = 0, any = 0;
    h266_chroma_res_block t{};
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint32_t xx = x + j;
      const uint32_t o = xx >= x0 && xx < x1 ? orow[xx >> c.sh] : 0;
      if (!o) continue;
      if (o != last) {
        t = b[o - 1];
        last = o;
      }
      if (!v16) v[j] = s[j];
      v[j] = res_add(v[j], res[t.res_offset + (uint64_t)(y - t.y) * t.w + (xx - t.x)], t.var_scale, lo, hi);
      if (!v16) s[j] = v[j];
      any = 1;
    }
    if (v16 && any) {
      uint32_t wd[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) wd[j] = (uint32_t)v[2 * j] | ((uint32_t)v[2 * j + 1] << 16);
      *reinterpret_cast<uint4 *>(s) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
    }
  }
  __syncthreads();
  if (live && ((y - y0) & ((1u << c.sh) - 1)) == 0) {  // the top row of each grid row clears it
    const uint32_t lo = max(x, x0) >> c.sh, hi = (min(x + 8, x1) - 1) >> c.sh;
    for (uint32_t cx = lo; cx <= hi; ++cx)
      if (orow[cx]) orow[cx] = 0;
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

int launch_lmcs_fwd_cover(cudaStream_t st, DPlane p, const uint16_t *d_lut, const RectPiece *d_pieces, uint32_t n,
                          const FwdCover &c, bool check, uint32_t *d_err, uint64_t *launches) {
  if (!n || c.x1 <= c.x0 || c.y1 <= c.y0) return H266_OK;
  const uint64_t warps = n;
  k_lmcs_fwd_count<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, st>>>(d_pieces, n, c);
  H266_CUDA(cudaGetLastError());
  const uint32_t tpr = (c.x1 - (c.x0 & ~7u) + 7) / 8;
  const dim3 grid((tpr + 31) / 32, (c.y1 - c.y0 + kBoxRows - 1) / kBoxRows);
  const int vec = ((uintptr_t)p.s & 15) == 0 && (p.stride & 7) == 0;
  k_lmcs_fwd_apply<<<grid, dim3(32, kBoxRows), 0, st>>>(p, d_lut, c, check ? 1 : 0, vec, d_err);
  H266_CUDA(cudaGetLastError());
  *launches += 2;
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
  k_chroma_residual<<<(n + kResWarps - 1) / kResWarps, kResWarps * 32, 0, st>>>(cb, cr, d_pieces, n, d_res, bd);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

int launch_chroma_residual_cover(cudaStream_t st, DPlane cb, DPlane cr, const h266_chroma_res_block *d_blocks,
                                 uint32_t n, const int32_t *d_res, int bd, const ResCover &c, uint32_t *d_overlap,
                                 uint64_t *launches) {
  if (!n) return H266_OK;
  k_res_own<<<(unsigned)(((uint64_t)n * 32 + 255) / 256), 256, 0, st>>>(d_blocks, n, c, d_overlap);
  H266_CUDA(cudaGetLastError());
  uint32_t gx = 0, gy = 0;
  for (int pl = 0; pl < 2; ++pl) {
    if (c.x1[pl] <= c.x0[pl] || c.y1[pl] <= c.y0[pl]) continue;
    gx = std::max(gx, ((c.x1[pl] - (c.x0[pl] & ~7u) + 7) / 8 + 31) / 32);
    gy = std::max(gy, (c.y1[pl] - c.y0[pl] + kBoxRows - 1) / kBoxRows);
  }
  ++*launches;
  if (!gx) return H266_OK;
  const int vec = ((uintptr_t)cb.s & 15) == 0 && (cb.stride & 7) == 0 && ((uintptr_t)cr.s & 15) == 0 &&
                  (cr.stride & 7) == 0;
  k_res_apply<<<dim3(gx, gy, 2), dim3(32, kBoxRows), 0, st>>>(cb, cr, d_blocks, d_res, c, bd, vec, d_overlap);
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
