// Encoder chroma ALF / CC-ALF trials (src/alf_enc.rs:628-1138): the per-CTB
// pieces around the trial passes.  Each trial is one run of the chain's
// SAO/ALF tile kernel (the candidate on every CTB, output into its own
// chroma plane); these kernels then sum the squared chroma error per CTB
// (ctb_sse_chroma, src/alf_enc.rs:823-849), pick per CTB the first minimum of
// {off, trial 0, ...} and copy the chosen trial's CTB samples into the
// reconstruction.
#include "internal.h"

namespace h266 {
namespace {

constexpr int kSseThreads = 256;

// One CTA per CTB: the SSE of `a` against `b` over the CTB's chroma region,
// rows and columns limited to both planes (the crate's early `break`s).
__global__ void __launch_bounds__(kSseThreads) k_ctb_sse(DPlane a, DPlane b, int cw, int ch, int w_ctbs,
                                                         unsigned long long *__restrict__ sse, int cols, int col) {
  const int i = blockIdx.x, rx = i % w_ctbs, ry = i / w_ctbs;
  const int x0 = rx * cw, y0 = ry * ch;
  const int x1 = min(x0 + cw, min(a.w, b.w)), y1 = min(y0 + ch, min(a.h, b.h));
  unsigned long long e = 0;
  if (x1 > x0 && y1 > y0) {
    const int w = x1 - x0;
    for (int y = y0 + threadIdx.x / 32; y < y1; y += kSseThreads / 32)
      for (int x = x0 + (threadIdx.x & 31); x < x0 + w; x += 32) {
        const int d = (int)a.s[(int64_t)y * a.stride + x] - (int)b.s[(int64_t)y * b.stride + x];
        e += (unsigned long long)((long long)d * d);
      }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
  __shared__ unsigned long long part[kSseThreads / 32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x / 32] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int k = 0; k < kSseThreads / 32; ++k) t += part[k];
    sse[(size_t)i * cols + col] = t;
  }
}

__global__ void k_trial_pick(const unsigned long long *__restrict__ sse, int cols, int n, int8_t *__restrict__ pick) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long *row = sse + (size_t)i * cols;
  unsigned long long best = row[0];
  int p = -1;
  for (int t = 1; t < cols; ++t)
    if (row[t] < best) {
      best = row[t];
      p = t - 1;
    }
  pick[i] = (int8_t)p;
}

// One CTA per CTB: copies the chosen trial's samples of the CTB region
// (clipped to the plane) into `dst`.
__global__ void __launch_bounds__(kSseThreads) k_ctb_commit(DPlane dst, const uint16_t *__restrict__ trials,
                                                            int64_t trial_samples, int trial_pitch, int cw, int ch,
                                                            int w_ctbs, const int8_t *__restrict__ pick) {
  const int i = blockIdx.x, p = pick[i];
  if (p < 0) return;
  const int rx = i % w_ctbs, ry = i / w_ctbs;
  const int x0 = rx * cw, y0 = ry * ch, x1 = min(x0 + cw, dst.w), y1 = min(y0 + ch, dst.h);
  const uint16_t *t = trials + (int64_t)p * trial_samples;
  for (int y = y0 + threadIdx.x / 32; y < y1; y += kSseThreads / 32)
    for (int x = x0 + (threadIdx.x & 31); x < x1; x += 32)
      dst.s[(int64_t)y * dst.stride + x] = t[(int64_t)y * trial_pitch + x];
}

}  // namespace

int launch_ctb_sse(cudaStream_t st, DPlane a, DPlane b, int cw, int ch, int w_ctbs, int n, unsigned long long *d_sse,
                   int cols, int col, uint64_t *launches) {
  if (n <= 0) return H266_OK;
  k_ctb_sse<<<n, kSseThreads, 0, st>>>(a, b, cw, ch, w_ctbs, d_sse, cols, col);
  H266_CUDA(cudaGetLastError());
  ++*launches;
  return H266_OK;
}

int launch_trial_pick_commit(cudaStream_t st, const unsigned long long *d_sse, int cols, int n, int8_t *d_pick,
                             DPlane dst, const uint16_t *d_trials, int64_t trial_samples, int trial_pitch, int cw,
                             int ch, int w_ctbs, uint64_t *launches) {
  if (n <= 0) return H266_OK;
  k_trial_pick<<<(n + 127) / 128, 128, 0, st>>>(d_sse, cols, n, d_pick);
  H266_CUDA(cudaGetLastError());
  k_ctb_commit<<<n, kSseThreads, 0, st>>>(dst, d_trials, trial_samples, trial_pitch, cw, ch, w_ctbs, d_pick);
  H266_CUDA(cudaGetLastError());
  *launches += 2;
  return H266_OK;
}

}  // namespace h266
