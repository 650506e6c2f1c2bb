// C ABI of the filter chain: contexts, argument validation, side-information
// packing and the per-filter / whole-chain entry points declared in
// include/oxideav_h266_b200.h.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>

#include "fixed_filters.h"
#include "internal.h"

static_assert(sizeof(h266_plane) == 32, "h266_plane");
static_assert(sizeof(h266_picture) == 104, "h266_picture");
static_assert(sizeof(h266_deblock_cu) == 96, "h266_deblock_cu");
static_assert(sizeof(h266_deblock_mv_cell) == 28, "h266_deblock_mv_cell");
static_assert(sizeof(h266_deblock_params) == 44, "h266_deblock_params");
static_assert(sizeof(h266_sao_ctb) == 24, "h266_sao_ctb");
static_assert(sizeof(h266_sao_ctb_params) == 72, "h266_sao_ctb_params");
static_assert(sizeof(h266_alf_ctb) == 8, "h266_alf_ctb");
static_assert(sizeof(h266_alf_aps_data) == 1992, "h266_alf_aps_data");
static_assert(sizeof(h266_lmcs_data) == 88, "h266_lmcs_data");
static_assert(sizeof(h266_lmcs_derived) == 400, "h266_lmcs_derived");
static_assert(sizeof(h266_in_loop_filter_args) == 256, "h266_in_loop_filter_args");

namespace h266 {

static thread_local std::string g_last_error;

int set_error(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

int cuda_error(cudaError_t e, const char *what) {
  const int code = e == cudaErrorMemoryAllocation ? H266_ERR_OUT_OF_MEMORY : H266_ERR_CUDA;
  return set_error(code, std::string(what) + ": " + cudaGetErrorString(e));
}

int DevBuf::ensure(size_t bytes) {
  if (bytes <= cap) return H266_OK;
  if (ptr) H266_CUDA(cudaDeviceSynchronize());  // queued work may still read the old allocation
  release();
  size_t want = std::max<size_t>(bytes, 256);
  want = want + want / 4;  // headroom against regrowth
  H266_CUDA(cudaMalloc(&ptr, want));
  cap = want;
  return H266_OK;
}

void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  cap = 0;
}

// Pinned host staging for one side-information upload per call.
struct Staging {
  uint8_t *ptr = nullptr;
  size_t cap = 0, used = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return H266_OK;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    size_t want = bytes + bytes / 4 + 4096;
    H266_CUDA(cudaHostAlloc((void **)&ptr, want, cudaHostAllocDefault));
    cap = want;
    return H266_OK;
  }
};

// Device scratch that the kernels using it hand back in its resting state
// (counters at zero, owners cleared): filled on allocation and after a call
// that did not complete, not on every call.
struct CleanBuf {
  DevBuf buf;
  bool clean = false;
  // Room for `bytes`, resting (all zero) on the stream; resting again only
  // once the caller reports a completed call with done().
  int ensure(size_t bytes, cudaStream_t st) {
    const size_t cap = buf.cap;
    H266_TRY(buf.ensure(bytes));
    if (buf.cap != cap) clean = false;
    if (!clean) H266_CUDA(cudaMemsetAsync(buf.ptr, 0, buf.cap, st));
    clean = false;
    return H266_OK;
  }
  void done() { clean = true; }
  void release() {
    buf.release();
    clean = false;
  }
};

}  // namespace h266

using namespace h266;

namespace h266 {
// One stream's worth of chain resources.  The context's main lane runs the
// single-picture calls on the context stream; batch calls spread pictures over
// extra lanes with their own streams so that the uploads, kernels and
// downloads of successive pictures overlap.
struct Lane {
  cudaStream_t stream = nullptr;
  bool owns_stream = false;
  cudaEvent_t staged = nullptr;  // last side-information upload done reading the staging buffer
  cudaEvent_t mark = nullptr;    // joins this lane with other streams
  DevBuf io[3];       // device copies of host pictures
  DevBuf scratch[3];  // deblocked planes read by the SAO / ALF pass
  DevBuf lut;         // LMCS inverse LUT
  DevBuf fwd_lut;     // LMCS forward LUT of fwd_key (valid when fwd_ok)
  h266_lmcs_derived fwd_key{};
  bool fwd_ok = false;
  CleanBuf fwd_cover;  // forward map: error word, then the coverage counters
  CleanBuf res_cover;  // residual add: overlap word, then the Cb and Cr cell owners
  DevBuf side;        // side information
  DevBuf walk;        // CU maps and segment grids of device-built side information
  Staging stage;
  int init(cudaStream_t s) {
    if (!s) {
      H266_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
      owns_stream = true;
    } else {
      stream = s;
    }
    H266_CUDA(cudaEventCreateWithFlags(&staged, cudaEventDisableTiming));
    H266_CUDA(cudaEventCreateWithFlags(&mark, cudaEventDisableTiming));
    H266_CUDA(cudaEventRecord(staged, stream));
    return H266_OK;
  }
  void release() {
    for (int i = 0; i < 3; ++i) {
      io[i].release();
      scratch[i].release();
    }
    lut.release();
    fwd_lut.release();
    fwd_ok = false;
    fwd_cover.release();
    res_cover.release();
    side.release();
    walk.release();
    if (stage.ptr) cudaFreeHost(stage.ptr);
    stage.ptr = nullptr;
    stage.cap = 0;
    if (staged) cudaEventDestroy(staged);
    if (mark) cudaEventDestroy(mark);
    staged = mark = nullptr;
    if (owns_stream && stream) cudaStreamDestroy(stream);
    stream = nullptr;
  }
};

struct Prep;  // host-side preparation of one picture's chain call

// Parameter tables of batched plan executions: assembled on the host,
// uploaded once per batch through pinned staging.
struct BatchBufs {
  bool capturing = false;  // recorded into a CUDA graph: no waits on events from outside the capture
  std::vector<uint8_t> blob;
  DevBuf side;
  Staging stage;
  cudaEvent_t staged = nullptr;  // the last upload has read the staging buffer
  cudaEvent_t done = nullptr;    // the last batch that reads `side` has finished its launches
  int init() {
    if (!staged) H266_CUDA(cudaEventCreateWithFlags(&staged, cudaEventDisableTiming));
    if (!done) H266_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    return H266_OK;
  }
  void release() {
    side.release();
    if (stage.ptr) cudaFreeHost(stage.ptr);
    stage.ptr = nullptr;
    stage.cap = 0;
    if (staged) cudaEventDestroy(staged);
    if (done) cudaEventDestroy(done);
    staged = done = nullptr;
  }
};

// One stream of the end-to-end batch pipeline (h266_apply_in_loop_filters_batch):
// device buffers for a group of pictures -- copies of host planes, deblocked
// planes, LMCS LUT, side information, walk scratch -- and the parameter tables
// of the group's batched launches.  Groups rotate over the lanes, so one
// group's uploads, another's kernels and a third one's downloads overlap.
struct GroupSlot {
  DevBuf io[3], scratch[3], lut, side, walk;
  void release() {
    for (int i = 0; i < 3; ++i) {
      io[i].release();
      scratch[i].release();
    }
    lut.release();
    side.release();
    walk.release();
  }
};
// Launch-shape knobs (h266_ctx_set_tuning); -1 in an override: not set.
struct Tuning {
  int e2e_group = 4, e2e_lanes = 4, sao_alf_ctas_per_sm = 0, sao_alf_tile_h = 64;
  int prep_threads = 0;  // 0: the default count
  // 1: every upload of the end-to-end batch (planes, side information, batch
  // tables) in issue order on one stream and every download on another, so
  // small latency-critical copies do not wait behind other lanes' planes in
  // the copy engine (measured 9.0 against 10.3 ms per 32 x 1080p)
  int e2e_copy_streams = 1;
  int e2e_ramp = 1;  // 1: the end-to-end batch starts and ends with groups of 1, 2, ... pictures
};
struct TuningKey {
  const char *name;
  int Tuning::*field;
  int lo, hi;
};
constexpr TuningKey kTuningKeys[] = {{"e2e_group", &Tuning::e2e_group, 1, 16},
                                     {"e2e_lanes", &Tuning::e2e_lanes, 1, 16},
                                     {"sao_alf_ctas_per_sm", &Tuning::sao_alf_ctas_per_sm, 0, 4},
                                     {"sao_alf_tile_h", &Tuning::sao_alf_tile_h, 32, 64},
                                     {"prep_threads", &Tuning::prep_threads, 0, 64},
                                     {"e2e_copy_streams", &Tuning::e2e_copy_streams, 0, 1},
                                     {"e2e_ramp", &Tuning::e2e_ramp, 0, 1}};

struct GroupLane {
  cudaStream_t stream = nullptr;
  cudaEvent_t mark = nullptr;
  // with separate copy streams: the group's uploads done, its kernels done,
  // its downloads done (the slots are free again)
  cudaEvent_t ev_up = nullptr, ev_comp = nullptr, ev_down = nullptr;
  std::vector<GroupSlot> slots;
  BatchBufs bb;
  int init(size_t n_slots) {
    H266_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    H266_CUDA(cudaEventCreateWithFlags(&mark, cudaEventDisableTiming));
    H266_CUDA(cudaEventCreateWithFlags(&ev_up, cudaEventDisableTiming));
    H266_CUDA(cudaEventCreateWithFlags(&ev_comp, cudaEventDisableTiming));
    H266_CUDA(cudaEventCreateWithFlags(&ev_down, cudaEventDisableTiming));
    slots.resize(n_slots);
    return bb.init();
  }
  void release() {
    if (stream) cudaStreamSynchronize(stream);
    for (GroupSlot &sl : slots) sl.release();
    bb.release();
    for (cudaEvent_t *e : {&mark, &ev_up, &ev_comp, &ev_down})
      if (*e) cudaEventDestroy(*e), *e = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
  }
};
}  // namespace h266

struct h266_ctx {
  int device = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  uint64_t launches = 0;
  uint64_t h2d_bytes = 0, d2h_bytes = 0;  // host <-> device copies queued by the context
  h266::Lane main;                                   // single-picture calls (stream = ctx->stream)
  std::vector<std::unique_ptr<h266::Lane>> lanes;    // batch calls
  std::unique_ptr<h266::TaskPool> pool;              // host side-information builders
  std::vector<std::unique_ptr<h266::Prep>> preps;    // [0]: single-picture calls, [i]: batch picture i
  // profiling: CUDA events around every launch, resolved in h266_ctx_profile
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;
  double prof_ms[H266_PROF_FAMILIES] = {0};
  // host time of h266_apply_in_loop_filters_batch (h266_ctx_host_profile):
  // preparation summed over workers, the issuing thread waiting for it, issuing
  std::atomic<int64_t> host_ns[3] = {{0}, {0}, {0}};
  uint64_t prof_n[H266_PROF_FAMILIES] = {0};
  h266::BatchBufs batch;  // parameter tables of h266_chain_plan_execute_batch
  std::vector<h266::RectPiece> fwd_pieces;  // forward-map pieces (capacity kept between calls)
  std::vector<h266::ResPiece> res_pieces;   // residual-add pieces (capacity kept between calls)
  std::vector<std::unique_ptr<h266::GroupLane>> glanes;  // the end-to-end batch pipeline
  cudaStream_t e2e_up = nullptr, e2e_down = nullptr;      // its copy streams
  bool force_scalar = false;  // H266_FORCE_SCALAR_ALF=1: scalar SAO/ALF kernel (cross-checks)
  bool force_global_deblock = false;  // H266_FORCE_GLOBAL_DEBLOCK=1: deblocking on global memory (cross-checks)
  bool force_strip_deblock = false;   // H266_FORCE_STRIP_DEBLOCK=1: strip kernels instead of tiles (cross-checks)
  bool force_host_sideinfo = false;   // H266_FORCE_HOST_SIDEINFO=1: never build side information on the device
  // launch-shape tuning (h266_ctx_set_tuning): context values and per-geometry overrides
  h266::Tuning tuning;
  std::map<uint64_t, h266::Tuning> tuning_for;  // key: width << 32 | height << 8 | bit depth
};

namespace {

struct Guard {  // makes the context's device current for the call
  int prev = -1;
  explicit Guard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~Guard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Brackets a launch with profiling events when profiling is on.
struct Prof {
  h266_ctx *ctx;
  cudaStream_t st;
  int fam;
  cudaEvent_t a = nullptr;
  static cudaEvent_t take(h266_ctx *c) {
    if (!c->ev_pool.empty()) {
      cudaEvent_t e = c->ev_pool.back();
      c->ev_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
  Prof(h266_ctx *c, cudaStream_t stream, int family) : ctx(c), st(stream), fam(family) {
    if (ctx->prof) {
      a = take(ctx);
      cudaEventRecord(a, st);
    }
  }
  ~Prof() {
    if (a) {
      cudaEvent_t b = take(ctx);
      cudaEventRecord(b, st);
      ctx->ev_pending.push_back({fam, {a, b}});
    }
  }
};

int check_ctx(h266_ctx *ctx) { return ctx ? H266_OK : set_error(H266_ERR_INVALID_ARGUMENT, "NULL context"); }

int check_picture(const h266_picture *pic) {
  if (!pic) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL picture");
  if (pic->mem != H266_MEM_HOST && pic->mem != H266_MEM_DEVICE)
    return set_error(H266_ERR_INVALID_ARGUMENT, "picture.mem must be H266_MEM_HOST or H266_MEM_DEVICE");
  const h266_plane *pl[3] = {&pic->luma, &pic->cb, &pic->cr};
  for (int i = 0; i < 3; ++i) {
    const h266_plane &p = *pl[i];
    if (p.width > 65535 || p.height > 65535) return set_error(H266_ERR_UNSUPPORTED, "plane larger than 65535");
    if ((uint64_t)p.width * p.height == 0) continue;
    if (!p.samples) return set_error(H266_ERR_INVALID_ARGUMENT, "plane samples pointer is NULL");
    if (p.stride < p.width) return set_error(H266_ERR_INVALID_ARGUMENT, "plane stride < width");
    if (p.bit_depth < 8 || p.bit_depth > 16) return set_error(H266_ERR_INVALID_ARGUMENT, "plane bit_depth must be 8..16");
  }
  if ((uint64_t)pic->luma.width * pic->luma.height == 0)
    return set_error(H266_ERR_INVALID_ARGUMENT, "empty luma plane");
  return H266_OK;
}

DPlane dplane(const h266_plane &p, uint16_t *ptr, int64_t stride) {
  return DPlane{ptr, stride, (int)p.width, (int)p.height};
}

// Device views of the picture: the caller's planes (device memory) or the
// context's copies of them (host memory, uploaded here).
uint64_t host_plane_bytes(const h266_picture &pic) {  // bytes of the planes of a host picture
  if (pic.mem != H266_MEM_HOST) return 0;
  const h266_plane *pl[3] = {&pic.luma, &pic.cb, &pic.cr};
  uint64_t b = 0;
  for (const h266_plane *p : pl) b += (uint64_t)p->width * p->height * 2;
  return b;
}

int picture_to_device(Lane &ln, const h266_picture &pic, DPlane out[3]) {
  const h266_plane *pl[3] = {&pic.luma, &pic.cb, &pic.cr};
  for (int i = 0; i < 3; ++i) {
    const h266_plane &p = *pl[i];
    const bool empty = (uint64_t)p.width * p.height == 0;
    if (pic.mem == H266_MEM_DEVICE || empty) {
      out[i] = dplane(p, p.samples, (int64_t)std::max<uint64_t>(p.stride, 1));
      continue;
    }
    const size_t row = (size_t)p.width * 2;
    H266_TRY(ln.io[i].ensure(row * p.height));
    H266_CUDA(cudaMemcpy2DAsync(ln.io[i].ptr, row, p.samples, (size_t)p.stride * 2, row, p.height,
                                cudaMemcpyHostToDevice, ln.stream));
    out[i] = dplane(p, ln.io[i].as<uint16_t>(), p.width);
  }
  return H266_OK;
}

// Queues the copies of a host picture back from the lane; with `sync` waits
// for them.
int picture_from_device(Lane &ln, const h266_picture &pic, bool sync = true) {
  if (pic.mem == H266_MEM_DEVICE) return H266_OK;
  const h266_plane *pl[3] = {&pic.luma, &pic.cb, &pic.cr};
  for (int i = 0; i < 3; ++i) {
    const h266_plane &p = *pl[i];
    if ((uint64_t)p.width * p.height == 0) continue;
    const size_t row = (size_t)p.width * 2;
    H266_CUDA(cudaMemcpy2DAsync(p.samples, (size_t)p.stride * 2, ln.io[i].ptr, row, row, p.height,
                                cudaMemcpyDeviceToHost, ln.stream));
  }
  if (sync) H266_CUDA(cudaStreamSynchronize(ln.stream));
  return H266_OK;
}

// ---------------------------------------------------------------- side-information blob
struct Blob {
  std::vector<uint8_t> &b;
  size_t put(const void *p, size_t n) {  // 256-byte aligned sections
    size_t off = (b.size() + 255) & ~(size_t)255;
    b.resize(off + n);
    if (n) std::memcpy(b.data() + off, p, n);
    return off;
  }
  // A section of n bytes for the caller to fill (before the next put / alloc).
  uint8_t *alloc(size_t n, size_t &off) {
    off = (b.size() + 255) & ~(size_t)255;
    b.resize(off + n);
    return b.data() + off;
  }
};

int upload_blob(Lane &ln, const std::vector<uint8_t> &blob, uint8_t **dev_base) {
  const size_t n = blob.size();
  H266_TRY(ln.side.ensure(n));
  H266_CUDA(cudaEventSynchronize(ln.staged));  // previous upload finished reading the staging buffer
  H266_TRY(ln.stage.ensure(n));
  std::memcpy(ln.stage.ptr, blob.data(), n);
  H266_CUDA(cudaMemcpyAsync(ln.side.ptr, ln.stage.ptr, n, cudaMemcpyHostToDevice, ln.stream));
  H266_CUDA(cudaEventRecord(ln.staged, ln.stream));
  *dev_base = ln.side.as<uint8_t>();
  return H266_OK;
}

// The same from caller memory, copied once into the staging buffer.
int upload_raw(Lane &ln, const void *p, size_t n, uint8_t **dev_base) {
  H266_TRY(ln.side.ensure(std::max<size_t>(n, 1)));
  H266_CUDA(cudaEventSynchronize(ln.staged));
  H266_TRY(ln.stage.ensure(std::max<size_t>(n, 1)));
  if (n) {
    std::memcpy(ln.stage.ptr, p, n);
    H266_CUDA(cudaMemcpyAsync(ln.side.ptr, ln.stage.ptr, n, cudaMemcpyHostToDevice, ln.stream));
  }
  H266_CUDA(cudaEventRecord(ln.staged, ln.stream));
  *dev_base = ln.side.as<uint8_t>();
  return H266_OK;
}

// ---------------------------------------------------------------- pass-2 tables
void chroma_sub(uint32_t cfi, int &sw, int &sh) {  // SaoConfig / AlfConfig::chroma_subsampling
  sw = cfi == 1 || cfi == 2 ? 2 : 1;
  sh = cfi == 1 ? 2 : 1;
}

// `span` of apply_sao_clipped (src/sao.rs:429-436) / clip_rect_for_ctb (src/alf.rs:1084-1091)
void span(const uint32_t *b, uint64_t n, uint32_t v, int mx, int &lo, int &hi) {
  for (uint64_t i = 0; i + 1 < n; ++i)
    if (v >= b[i] && v < b[i + 1]) {
      lo = (int)b[i];
      hi = std::min((int)b[i + 1], mx);
      return;
    }
  lo = 0;
  hi = mx;
}

int alf_clip_value(int bd, int idx) {  // Table 8 (resolve_clip_value, src/alf.rs:627-644)
  static const int kDrop[4] = {0, 3, 5, 7};
  bd = std::min(std::max(bd, 8), 16);
  return 1 << (bd - kDrop[idx & 3]);
}

struct Pass2Inputs {
  const h266_sao_picture *sao = nullptr;
  const h266_sao_config *sao_cfg = nullptr;
  const h266_alf_picture *alf = nullptr;
  const h266_alf_config *alf_cfg = nullptr;
  const h266_alf_aps_binding *binding = nullptr;
  const uint32_t *cols = nullptr, *rows = nullptr;
  uint64_t n_cols = 0, n_rows = 0;
};

struct Pass2Host {
  std::vector<CtbDev> ctbs;
  std::vector<int32_t> luma_tab;      // slots * 600: coeff[300] then clip[300]
  std::vector<uint32_t> luma_packed;  // packed-arithmetic form, see AlfTablesDev
  Pass2Args args;
  bool do_sao = false, do_alf = false;
  bool packed = false;  // run the packed 16x2 kernel
};

// eqs. 1442-1445: coefficient / clip permutation per transposeIdx
const int kTranspose[4][12] = {{0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11},
                               {9, 4, 10, 8, 1, 5, 11, 7, 3, 0, 2, 6},
                               {0, 3, 2, 1, 8, 7, 6, 5, 4, 9, 10, 11},
                               {9, 8, 10, 4, 3, 7, 11, 5, 1, 0, 2, 6}};

// Builds the packed tables; returns false when an input is outside the packed
// path's range (then the scalar kernel runs).
bool build_packed(Pass2Host &h, int bd, uint32_t cfi, const h266_alf_aps_data *caps) {
  if (bd > 14 || (cfi != 0 && cfi != 1)) return false;
  auto in8 = [](int v) { return v >= -128 && v <= 127; };
  const size_t slots = h.luma_tab.size() / 600;
  h.luma_packed.assign(slots * 100 * 36, 0);
  for (size_t s = 0; s < slots; ++s)
    for (int c = 0; c < 25; ++c)
      for (int t = 0; t < 4; ++t)
        for (int k = 0; k < 12; ++k) {
          const int src = kTranspose[t][k];
          const int coef = h.luma_tab[s * 600 + c * 12 + src], clip = h.luma_tab[s * 600 + 300 + c * 12 + src];
          if (!in8(coef)) return false;
          uint32_t *w = &h.luma_packed[((s * 100) + c * 4 + t) * 36 + 3 * k];
          w[0] = ((uint32_t)clip & 0xFFFF) | ((uint32_t)clip << 16);
          w[1] = ((uint32_t)(-clip) & 0xFFFF) | ((uint32_t)(-clip) << 16);
          w[2] = ((uint32_t)coef & 0xFF) | ((uint32_t)coef & 0xFF) << 24;  // dp2a_lo: low lane, dp2a_hi: high lane
        }
  if (caps)
    for (uint32_t f = 0; f < caps->n_chroma_filters; ++f)
      for (int k = 0; k < 6; ++k) {
        const int coef = caps->chroma_coeff[f][k], clip = alf_clip_value(bd, caps->chroma_clip_idx[f][k]);
        if (!in8(coef)) return false;
        uint32_t *w = &h.args.tables.chroma_packed[f * 18 + 3 * k];
        w[0] = ((uint32_t)clip & 0xFFFF) | ((uint32_t)clip << 16);
        w[1] = ((uint32_t)(-clip) & 0xFFFF) | ((uint32_t)(-clip) << 16);
        w[2] = ((uint32_t)coef & 0xFF) | ((uint32_t)coef & 0xFF) << 24;
      }
  // CC-ALF taps are applied as signed-byte dp2a weights
  for (int c = 0; c < 2; ++c)
    for (int f = 0; f < 4; ++f)
      for (int k = 0; k < 7; ++k)
        if (!in8(h.args.tables.cc_coeff[c][f][k])) return false;
  return true;
}

int check_bounds(const uint32_t *b, uint64_t n, uint32_t extent, uint32_t ctb, const char *what) {
  if (n && !b) return set_error(H266_ERR_INVALID_ARGUMENT, std::string(what) + ": NULL list");
  for (uint64_t i = 0; i < n; ++i)
    if (b[i] < extent && b[i] % ctb != 0)
      return set_error(H266_ERR_UNSUPPORTED, std::string(what) + ": clip bound not on the CTB grid");
  return H266_OK;
}

int build_pass2(const h266_picture &pic, const Pass2Inputs &in, Pass2Host &h) {
  Pass2Args &a = h.args;
  std::memset(&a, 0, sizeof a);
  const bool sao_on = in.sao && in.sao_cfg && (in.sao_cfg->luma_used || in.sao_cfg->chroma_used);
  const bool alf_on = in.alf && in.alf_cfg && in.alf_cfg->alf_enabled;
  h.do_sao = sao_on;
  h.do_alf = alf_on;
  if (!sao_on && !alf_on) return H266_OK;
  uint32_t bd = 0, log2 = 0, cfi = 0;
  if (sao_on) {
    bd = in.sao_cfg->bit_depth;
    log2 = in.sao_cfg->ctb_log2_size_y;
    cfi = in.sao_cfg->chroma_format_idc;
  }
  if (alf_on) {
    if (sao_on && (in.alf_cfg->bit_depth != bd || in.alf_cfg->ctb_log2_size_y != log2 ||
                   in.alf_cfg->chroma_format_idc != cfi))
      return set_error(H266_ERR_UNSUPPORTED, "SAO and ALF configs disagree on bit depth / CTB size / chroma format");
    bd = in.alf_cfg->bit_depth;
    log2 = in.alf_cfg->ctb_log2_size_y;
    cfi = in.alf_cfg->chroma_format_idc;
  }
  if (bd < 8 || bd > 16) return set_error(H266_ERR_INVALID_ARGUMENT, "SAO/ALF bit_depth must be 8..16");
  if (log2 < 5 || log2 > 7) return set_error(H266_ERR_UNSUPPORTED, "SAO/ALF need CtbLog2SizeY in 5..7");
  if (cfi > 3) return set_error(H266_ERR_INVALID_ARGUMENT, "chroma_format_idc must be 0..3");
  const uint32_t ctb = 1u << log2;
  H266_TRY(check_bounds(in.cols, in.n_cols, pic.luma.width, ctb, "clip cols"));
  H266_TRY(check_bounds(in.rows, in.n_rows, pic.luma.height, ctb, "clip rows"));
  uint32_t wc = 0, hc = 0;
  if (sao_on) {
    wc = in.sao->pic_width_in_ctbs_y;
    hc = in.sao->pic_height_in_ctbs_y;
    if ((uint64_t)wc * hc && !in.sao->ctbs) return set_error(H266_ERR_INVALID_ARGUMENT, "SaoPicture.ctbs is NULL");
  }
  if (alf_on) {
    if ((uint64_t)in.alf->pic_width_in_ctbs_y * in.alf->pic_height_in_ctbs_y && !in.alf->ctbs)
      return set_error(H266_ERR_INVALID_ARGUMENT, "AlfPicture.ctbs is NULL");
    if (sao_on && (in.alf->pic_width_in_ctbs_y != wc || in.alf->pic_height_in_ctbs_y != hc))
      return set_error(H266_ERR_GRID_MISMATCH, "SaoPicture and AlfPicture CTB grids differ");
    wc = in.alf->pic_width_in_ctbs_y;
    hc = in.alf->pic_height_in_ctbs_y;
  }
  if ((uint64_t)wc * hc > (1u << 24)) return set_error(H266_ERR_UNSUPPORTED, "CTB grid too large");
  int sw, sh;
  chroma_sub(cfi, sw, sh);
  const int pw = (int)pic.luma.width, ph = (int)pic.luma.height;
  const bool chroma = cfi != 0 && (uint64_t)pic.cb.width * pic.cb.height + (uint64_t)pic.cr.width * pic.cr.height > 0;
  if (chroma) {  // PictureBuffer chroma is floor or ceil of luma / SubWidthC (src/reconstruct.rs:130-139)
    const h266_plane *cp[2] = {&pic.cb, &pic.cr};
    for (const h266_plane *c : cp) {
      if ((uint64_t)c->width * c->height == 0) continue;
      const uint32_t fw = pic.luma.width / sw, cw = (pic.luma.width + sw - 1) / sw;
      const uint32_t fh = pic.luma.height / sh, ch = (pic.luma.height + sh - 1) / sh;
      if (c->width < fw || c->width > cw || c->height < fh || c->height > ch)
        return set_error(H266_ERR_UNSUPPORTED, "chroma plane size does not match the luma size and chroma format");
    }
  }
  const h266_alf_aps_binding *b = in.binding;
  const h266_alf_aps_data *caps = (alf_on && b) ? b->chroma_aps : nullptr;
  const h266_alf_aps_data *ccaps[2] = {(alf_on && b) ? b->cc_cb_aps : nullptr, (alf_on && b) ? b->cc_cr_aps : nullptr};
  if (caps && caps->n_chroma_filters > 8) return set_error(H266_ERR_INVALID_ARGUMENT, "chroma APS: more than 8 filters");
  if (ccaps[0] && ccaps[0]->n_cc_cb_filters > 4) return set_error(H266_ERR_INVALID_ARGUMENT, "CC-ALF Cb: more than 4 filters");
  if (ccaps[1] && ccaps[1]->n_cc_cr_filters > 4) return set_error(H266_ERR_INVALID_ARGUMENT, "CC-ALF Cr: more than 4 filters");
  h.ctbs.assign((size_t)wc * hc, CtbDev{});
  h.luma_tab.clear();
  std::map<int, int> slot_of;  // luma_filt_set_idx -> compact slot, -1 = unresolved
  for (uint32_t ry = 0; ry < hc; ++ry)
    for (uint32_t rx = 0; rx < wc; ++rx) {
      CtbDev &d = h.ctbs[(size_t)ry * wc + rx];
      std::memset(&d, 0, sizeof d);
      d.luma_set = -1;
      d.chroma_filt[0] = d.chroma_filt[1] = -1;
      d.cc_filt[0] = d.cc_filt[1] = -1;
      int r[4] = {0, 0, pw, ph};
      if (in.cols) {
        span(in.cols, in.n_cols, rx * ctb, pw, r[0], r[2]);
        span(in.rows, in.n_rows, ry * ctb, ph, r[1], r[3]);
      }
      for (int k = 0; k < 4; ++k) d.rect[k] = (uint16_t)r[k];
      if (sao_on) {
        const h266_sao_ctb_params &s = in.sao->ctbs[(size_t)ry * wc + rx];
        const h266_sao_ctb *src[3] = {&s.luma, &s.cb, &s.cr};
        for (int c = 0; c < 3; ++c) {
          const bool used = c == 0 ? in.sao_cfg->luma_used != 0 : (in.sao_cfg->chroma_used && cfi != 0);
          const h266_sao_ctb &sc = *src[c];
          if (!used || (sc.sao_type_idx != 1 && sc.sao_type_idx != 2)) continue;
          d.sao[c].type = sc.sao_type_idx;
          d.sao[c].eo_class = sc.eo_class & 3;
          d.sao[c].band_pos = sc.band_position;
          for (int k = 0; k < 4; ++k) {
            if (sc.offset_val[k + 1] < -32768 || sc.offset_val[k + 1] > 32767)
              return set_error(H266_ERR_UNSUPPORTED, "SAO offset outside int16");
            d.sao[c].off[k] = (int16_t)sc.offset_val[k + 1];
          }
        }
      }
      if (alf_on) {
        const h266_alf_ctb &p = in.alf->ctbs[(size_t)ry * wc + rx];
        if (p.luma_on) {  // resolve_luma_filter_set, src/alf.rs:564-595
          const int idx = p.luma_filt_set_idx;
          auto it = slot_of.find(idx);
          int slot = -1;
          if (it != slot_of.end()) {
            slot = it->second;
          } else {
            const h266_alf_aps_data *aps = nullptr;
            bool ok = idx < 16;
            if (!ok && b && (uint32_t)(idx - 16) < b->n_luma_apses && b->luma_apses && b->luma_apses[idx - 16]) {
              aps = b->luma_apses[idx - 16];
              ok = aps->alf_luma_filter_signal_flag != 0;
              if (ok && aps->n_luma_filters < 25)
                return set_error(H266_ERR_INVALID_ARGUMENT, "luma APS signals fewer than 25 filters");
            }
            if (ok) {
              slot = (int)(h.luma_tab.size() / 600);
              h.luma_tab.resize(h.luma_tab.size() + 600);
              int32_t *t = &h.luma_tab[(size_t)slot * 600];
              for (int c = 0; c < 25; ++c)
                for (int j = 0; j < 12; ++j) {
                  t[c * 12 + j] = idx < 16 ? kFixedSetCoeff[(idx * 25 + c) * 12 + j] : aps->luma_coeff[c][j];
                  t[300 + c * 12 + j] = alf_clip_value((int)bd, idx < 16 ? 0 : aps->luma_clip_idx[c][j]);
                }
            }
            slot_of[idx] = slot;
          }
          d.luma_set = (int16_t)slot;
        }
        if (chroma) {
          const uint32_t en[2] = {in.alf_cfg->cb_enabled && p.cb_on, in.alf_cfg->cr_enabled && p.cr_on};
          const uint8_t alt[2] = {p.cb_alt_idx, p.cr_alt_idx};
          for (int c = 0; c < 2; ++c)
            if (en[c] && caps && caps->alf_chroma_filter_signal_flag && alt[c] < caps->n_chroma_filters)
              d.chroma_filt[c] = (int8_t)alt[c];
          const uint32_t cen[2] = {in.alf_cfg->cc_cb_enabled && p.cc_cb_idc != 0,
                                   in.alf_cfg->cc_cr_enabled && p.cc_cr_idc != 0};
          const uint8_t idc[2] = {p.cc_cb_idc, p.cc_cr_idc};
          for (int c = 0; c < 2; ++c) {
            if (!cen[c] || !ccaps[c]) continue;
            const uint32_t n = c == 0 ? ccaps[c]->n_cc_cb_filters : ccaps[c]->n_cc_cr_filters;
            if ((uint32_t)(idc[c] - 1) < n) d.cc_filt[c] = (int8_t)(idc[c] - 1);
          }
        }
      }
    }
  if (caps)
    for (uint32_t f = 0; f < caps->n_chroma_filters; ++f)
      for (int k = 0; k < 6; ++k) {
        a.tables.chroma_coeff[f][k] = caps->chroma_coeff[f][k];
        a.tables.chroma_clip[f][k] = alf_clip_value((int)bd, caps->chroma_clip_idx[f][k]);
      }
  for (int c = 0; c < 2; ++c)
    if (ccaps[c])
      for (int f = 0; f < 4; ++f)
        for (int k = 0; k < 7; ++k) a.tables.cc_coeff[c][f][k] = c == 0 ? ccaps[c]->cc_cb_coeff[f][k] : ccaps[c]->cc_cr_coeff[f][k];
  a.bit_depth = (int)bd;
  a.ctb_log2 = (int)log2;
  a.sub_w = sw;
  a.sub_h = sh;
  a.chroma = chroma ? 1 : 0;
  a.w_ctbs = (int)wc;
  a.h_ctbs = (int)hc;
  a.pic_w = pw;
  a.pic_h = ph;
  a.ext_w = std::max<int>(pw, (int)pic.cb.width * sw);
  a.ext_w = std::max<int>(a.ext_w, (int)pic.cr.width * sw);
  a.ext_h = std::max<int>(ph, (int)pic.cb.height * sh);
  a.ext_h = std::max<int>(a.ext_h, (int)pic.cr.height * sh);
  a.tiles_x = (a.ext_w + 31) / 32;
  a.tiles_y = (a.ext_h + 31) / 32;
  a.has_clip = in.cols != nullptr;
  a.sao_luma = sao_on && in.sao_cfg->luma_used;
  a.sao_chroma = sao_on && in.sao_cfg->chroma_used && cfi != 0;
  a.sao_i8 = 1;  // the packed SAO step looks offsets up as signed bytes
  for (const CtbDev &d : h.ctbs)
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 4; ++k)
        if (d.sao[c].off[k] < -128 || d.sao[c].off[k] > 127) a.sao_i8 = 0;
  h.packed = build_packed(h, (int)bd, cfi, caps);
  if (!h.packed) h.luma_packed.clear();
  return H266_OK;
}

// Side information of one call, assembled into one host blob and uploaded once.
struct Staged {
  size_t ctb = 0, tab = 0, pack = 0, seg[2] = {0, 0}, comp[2] = {0, 0}, band[2] = {0, 0};
  size_t tile_bounds = 0;
  size_t dw_cus = 0, dw_ccus = 0, dw_mv = 0, dw_cols = 0, dw_rows = 0;  // device-walk inputs
  size_t dw_tails[2] = {0, 0};
  uint8_t *base = nullptr;
};

// Sizes of the staged deblocking plan.
struct DbSide {
  uint32_t n_comp[2] = {0, 0};
  uint32_t band_off[2][3] = {{0, 0, 0}, {0, 0, 0}};
  uint32_t n_bands[2][3] = {{0, 0, 0}, {0, 0, 0}};
  bool tiles_ok = false;
  uint32_t tiles_x = 0, tiles_y = 0;
  uint32_t tb_off[2][3] = {{0, 0, 0}, {0, 0, 0}};
  // side information built on the device: the walk's inputs (pointers are
  // rebased onto the uploaded blob when the chain runs)
  bool device_walk = false, dw_sep = false, dw_mv = false, dw_mv_cu = false;
  bool dw_tiles = false;  // device walk without chained footprints, out of place: the grid-mode tile kernel
  DeviceWalkIn dw{};
};

void stage_deblock(const DeblockPlan &pl, std::vector<uint8_t> &b, Staged &st, DbSide &db) {
  Blob blob{b};
  for (int d = 0; d < 2; ++d) {
    st.seg[d] = blob.put(pl.segs[d].data(), pl.segs[d].size() * sizeof(EdgeSeg));
    st.comp[d] = blob.put(pl.comp[d].data(), pl.comp[d].size() * sizeof(uint32_t));
    st.band[d] = blob.put(pl.band_first[d].data(), pl.band_first[d].size() * sizeof(uint32_t));
    db.n_comp[d] = (uint32_t)pl.comp[d].size() - 1;
    for (int p = 0; p < 3; ++p) {
      db.band_off[d][p] = pl.band_off[d][p];
      db.n_bands[d][p] = pl.n_bands[d][p];
    }
  }
  db.tiles_ok = pl.tiles_ok;
  db.tiles_x = pl.tiles_x;
  db.tiles_y = pl.tiles_y;
  if (pl.tiles_ok) {
    st.tile_bounds = blob.put(pl.tile_bounds.data(), pl.tile_bounds.size() * sizeof(uint32_t));
    for (int d = 0; d < 2; ++d)
      for (int p = 0; p < 3; ++p) db.tb_off[d][p] = pl.tb_off[d][p];
  }
}

void stage_pass2(const Pass2Host &h, std::vector<uint8_t> &b, Staged &st) {
  Blob blob{b};
  st.ctb = blob.put(h.ctbs.data(), h.ctbs.size() * sizeof(CtbDev));
  st.tab = blob.put(h.luma_tab.data(), h.luma_tab.size() * sizeof(int32_t));
  st.pack = blob.put(h.luma_packed.data(), h.luma_packed.size() * sizeof(uint32_t));
}

// Runs pass 2 (SAO and/or ALF) from `src` into the picture planes `dst`.
// Completes the pass-2 arguments with the planes and the staged tables.
void bind_pass2(Pass2Args &a, const uint8_t *base, const Staged &st, const DPlane src[3], const DPlane dst[3]) {
  for (int i = 0; i < 3; ++i) {
    a.src[i] = src[i];
    a.dst[i] = dst[i];
  }
  a.ctbs = reinterpret_cast<const CtbDev *>(base + st.ctb);
  a.tables.luma_coeff = reinterpret_cast<const int32_t *>(base + st.tab);  // per slot: coeff[300], clip[300]
  a.tables.luma_clip = a.tables.luma_coeff + 300;
  a.tables.luma_packed = reinterpret_cast<const uint32_t *>(base + st.pack);
  pass2_tma_maps(a);
}

int run_pass2(h266_ctx *ctx, cudaStream_t stream, Pass2Args a, bool do_sao, bool do_alf, bool packed,
              const uint8_t *base, const Staged &st, const DPlane src[3], const DPlane dst[3]) {
  bind_pass2(a, base, st, src, dst);
  Prof pf(ctx, stream, H266_PROF_SAO_ALF);
  if (packed && !ctx->force_scalar) return launch_pass2_packed(stream, a, do_sao, do_alf, &ctx->launches);
  return launch_pass2(stream, a, do_sao, do_alf, &ctx->launches);
}

int ensure_scratch(Lane &ln, const DPlane p[3], DPlane s[3]) {
  for (int i = 0; i < 3; ++i) {
    const size_t n = (size_t)std::max(p[i].w, 0) * std::max(p[i].h, 0);
    H266_TRY(ln.scratch[i].ensure(std::max<size_t>(n, 1) * 2));
    s[i] = DPlane{ln.scratch[i].as<uint16_t>(), std::max(p[i].w, 1), p[i].w, p[i].h};
  }
  return H266_OK;
}

int plane_map(h266_ctx *ctx, cudaStream_t stream, DPlane dst, DPlane src, const uint16_t *lut);

// Deblocking of the planes `src` into `dst` (the same planes for in-place
// filtering), luma mapped through the LMCS LUT `lut` first when given: the
// tile kernel when the plan has tile lists and dst is not src, else the
// shared-memory strip kernels when the planes fit them, else plane copies and
// one thread per component on global memory.
DeviceWalkIn device_walk_in(const uint8_t *base, const Staged &st, const DbSide &db);

int run_deblock(h266_ctx *ctx, cudaStream_t stream, const uint8_t *base, const Staged &st, const DbSide &db,
                const DPlane src[3], const DPlane dst[3], const uint16_t *lut, int bd, uint8_t *walk = nullptr) {
  if (db.device_walk) {  // side information built on the device, then the tile or strip kernels on its grids
    if (!walk) return set_error(H266_ERR_INVALID_ARGUMENT, "device-built side information without walk scratch");
    if (db.dw_tiles && !db.dw.tile_lists) return set_error(H266_ERR_UNSUPPORTED, "grid-mode tiles without tile lists");
    Prof pf(ctx, stream, H266_PROF_DEBLOCK);
    DeviceWalkOut out;
    H266_TRY(launch_device_walk(stream, device_walk_in(base, st, db), walk, out, &ctx->launches));
    const bool apart = src[0].s != dst[0].s && src[1].s != dst[1].s && src[2].s != dst[2].s;
    if (db.dw_tiles && apart) return launch_deblock_tiles_grid(stream, src, dst, lut, bd, out, &ctx->launches);
    return launch_deblock_strips_grid(stream, src, dst, lut, bd, out, &ctx->launches);
  }
  const StripSide v{reinterpret_cast<const EdgeSeg *>(base + st.seg[0]),
                    reinterpret_cast<const uint32_t *>(base + st.comp[0]),
                    reinterpret_cast<const uint32_t *>(base + st.band[0])};
  const StripSide h{reinterpret_cast<const EdgeSeg *>(base + st.seg[1]),
                    reinterpret_cast<const uint32_t *>(base + st.comp[1]),
                    reinterpret_cast<const uint32_t *>(base + st.band[1])};
  const bool separate = src[0].s != dst[0].s && src[1].s != dst[1].s && src[2].s != dst[2].s;
  if (!ctx->force_global_deblock && !ctx->force_strip_deblock && db.tiles_ok && separate) {
    Prof pf(ctx, stream, H266_PROF_DEBLOCK);
    return launch_deblock_tiles(stream, src, dst, lut, bd, v, h,
                                reinterpret_cast<const uint32_t *>(base + st.tile_bounds), db.tb_off, db.n_bands,
                                db.tiles_x, db.tiles_y, &ctx->launches);
  }
  if (!ctx->force_global_deblock && deblock_strips_fit(dst)) {
    Prof pf(ctx, stream, H266_PROF_DEBLOCK);
    return launch_deblock_strips(stream, src, dst, lut, bd, v, h, db.band_off, db.n_bands, &ctx->launches);
  }
  for (int i = 0; i < 3; ++i)
    if (src[i].s != dst[i].s || (i == 0 && lut))
      H266_TRY(plane_map(ctx, stream, dst[i], src[i], i == 0 ? lut : nullptr));
  Prof pf(ctx, stream, H266_PROF_DEBLOCK);
  return launch_deblock(stream, dst, bd, reinterpret_cast<const EdgeSeg *>(base + st.seg[0]),
                        reinterpret_cast<const uint32_t *>(base + st.comp[0]), db.n_comp[0],
                        reinterpret_cast<const EdgeSeg *>(base + st.seg[1]),
                        reinterpret_cast<const uint32_t *>(base + st.comp[1]), db.n_comp[1], &ctx->launches);
}

int plane_map(h266_ctx *ctx, cudaStream_t stream, DPlane dst, DPlane src, const uint16_t *lut) {
  Prof pf(ctx, stream, lut ? H266_PROF_LMCS : H266_PROF_COPY);
  return launch_plane_map(stream, dst, src, lut, &ctx->launches);
}

int build_lut(h266_ctx *ctx, cudaStream_t stream, uint16_t *lut, const h266_lmcs_derived &l, uint32_t mn,
              uint32_t mx) {
  Prof pf(ctx, stream, H266_PROF_LMCS);
  return launch_lmcs_lut(stream, lut, l, mn, mx, &ctx->launches);
}

int check_lmcs(const h266_lmcs_derived *l, uint32_t mn, uint32_t mx) {
  if (!l) return H266_OK;
  if (l->bit_depth < 8 || l->bit_depth > 16) return set_error(H266_ERR_INVALID_ARGUMENT, "LMCS bit_depth must be 8..16");
  if (mn > 15 || mx > 15) return set_error(H266_ERR_INVALID_ARGUMENT, "LMCS bin index out of range");
  return H266_OK;
}

}  // namespace

// Host-side preparation of one chain call: the deblocking plan, the pass-2
// tables and the side-information blob with its section offsets.  A failed
// preparation keeps its status and message (it may run on a worker thread).
struct h266::Prep {
  DeblockPlan plan;
  std::vector<uint8_t> blob;
  Pass2Host h;
  Staged st;
  DbSide db;
  int rc = H266_OK;
  std::string msg;
  // Batch pictures: the blob copied to pinned memory by the worker that built
  // it, uploaded from there; `uploaded` marks the end of the last upload.
  Staging pinned;
  cudaEvent_t uploaded = nullptr;
  bool staged_pinned = false;
  ~Prep() {
    if (pinned.ptr) cudaFreeHost(pinned.ptr);
    if (uploaded) cudaEventDestroy(uploaded);
  }
  // Copies the blob to `pinned` (waiting for the previous upload from it).
  int stage() {
    staged_pinned = false;
    if (!uploaded) H266_CUDA(cudaEventCreateWithFlags(&uploaded, cudaEventDisableTiming));
    H266_CUDA(cudaEventSynchronize(uploaded));
    H266_TRY(pinned.ensure(blob.size()));
    std::memcpy(pinned.ptr, blob.data(), blob.size());
    staged_pinned = true;
    return H266_OK;
  }
};

// A chain whose side information is resident on the device (h266_chain_plan_create).
struct h266_chain_plan {
  int device = 0;
  h266_picture geom{};  // plane sizes / bit depths the plan was built for
  h266::DevBuf side, lut, scratch[3];
  h266::DevBuf walk;  // CU maps and segment grids of the device walk (db.device_walk)
  bool lmcs = false, pass2 = false;
  int deblock_bd = 8;
  Staged st;  // section offsets inside `side` (base unset)
  DbSide db;
  h266::Pass2Args args{};
  bool do_sao = false, do_alf = false, packed = false;
};

namespace h266 {
// One picture of a batched chain execution: device planes P (filtered in
// place), scratch planes S, its staged side information (st.base set), the
// pass-2 arguments before binding, LUT and walk scratch.
struct BatchItem {
  DPlane P[3], S[3];
  Staged st;
  DbSide db;
  Pass2Args args;
  bool pass2 = false, do_sao = false, do_alf = false, packed = false;
  const uint16_t *lut = nullptr;
  int bd = 8;
  uint8_t *walk = nullptr;
};
int exec_batch(h266_ctx *ctx, BatchBufs &bb, cudaStream_t stream, std::vector<BatchItem> &items,
               const Tuning &tn, cudaStream_t upload = nullptr);
}  // namespace h266

// The tuning of a batch: the override for its largest picture's geometry, else the context's.
static const h266::Tuning &batch_tuning(const h266_ctx *ctx, uint32_t n, const h266_picture *const *pics) {
  uint64_t best = 0, px = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const h266_picture &p = *pics[i];
    const uint64_t a = (uint64_t)p.luma.width * p.luma.height;
    if (a > px) {
      px = a;
      best = (uint64_t)p.luma.width << 32 | (uint64_t)(p.luma.height & 0xFFFFFF) << 8 | (p.luma.bit_depth & 0xFF);
    }
  }
  const auto it = ctx->tuning_for.find(best);
  return it == ctx->tuning_for.end() ? ctx->tuning : it->second;
}



namespace {

// `allow_device`: a picture whose side information the device can build
// (device_walk_mode non-zero) skips the host walk; its CU lists, motion grid
// and gate lists are staged instead.  Pictures without chained footprints
// and with SAO or ALF on (deblocking out of place) deblock with the grid-mode
// tile kernel, the others with the grid-mode strip kernels.
int prepare_chain(Prep &pr, const h266_picture &pic, const h266_in_loop_filter_args &a, TaskPool *pool,
                  bool allow_device = false) {
  pr.st = Staged{};
  pr.db = DbSide{};
  pr.staged_pinned = false;
  H266_TRY(check_lmcs(a.lmcs, a.lmcs_min_bin_idx, a.lmcs_max_bin_idx));
  if ((a.n_cus && !a.cus) || (a.n_no_filter_cols && !a.no_filter_cols) || (a.n_no_filter_rows && !a.no_filter_rows))
    return set_error(H266_ERR_INVALID_ARGUMENT, "NULL list with nonzero length");
  if (a.clip_cols && !a.clip_rows) return set_error(H266_ERR_INVALID_ARGUMENT, "clip_rows is NULL while clip_cols is not");
  Pass2Inputs in;
  in.sao = a.sao;
  in.sao_cfg = a.sao ? &a.sao_cfg : nullptr;
  in.alf = a.alf;
  in.alf_cfg = a.alf ? &a.alf_cfg : nullptr;
  in.binding = a.alf_binding;
  in.cols = a.clip_cols;
  in.rows = a.clip_rows;
  in.n_cols = a.n_clip_cols;
  in.n_rows = a.n_clip_rows;
  H266_TRY(build_pass2(pic, in, pr.h));
  pr.blob.clear();
  const int mode = allow_device ? device_walk_mode(pic, a.cus, a.n_cus, a.chroma_cus, a.n_chroma_cus, a.deblock,
                                                   a.chroma_format_idc)
                                : 0;
  if (mode) {
    Blob blob{pr.blob};
    DbSide &db = pr.db;
    db.device_walk = true;
    db.dw_tiles = mode == 1 && (pr.h.do_sao || pr.h.do_alf);
    db.dw.tile_lists = mode == 1;  // the walk lists each tile's cells (within the lists' caps in mode 1)
    db.dw.tiles_consume = db.dw_tiles;
    db.dw_sep = a.chroma_cus != nullptr;
    db.dw_mv = a.mv_grid && a.mv_grid->cells && a.mv_grid->cells_w * a.mv_grid->cells_h;
    DeviceWalkIn &w = db.dw;
    w.n_cus = a.n_cus;
    w.n_chroma = db.dw_sep ? a.n_chroma_cus : 0;
    w.mv_w = db.dw_mv ? a.mv_grid->cells_w : 0;
    w.mv_h = db.dw_mv ? a.mv_grid->cells_h : 0;
    w.n_cols = a.n_no_filter_cols;
    w.n_rows = a.n_no_filter_rows;
    w.params = a.deblock;
    w.cfi = a.chroma_format_idc;
    w.w = (int)pic.luma.width;
    w.h = (int)pic.luma.height;
    w.sep = db.dw_sep;
    w.cw = (int)pic.cb.width;
    w.ch = (int)pic.cb.height;
    // the CU lists packed: every CU's head, the tails of CUs with a TU map or a TB split
    w.max_cu_dim = 4;
    const h266_deblock_cu *lists[2] = {a.cus, a.chroma_cus};
    const uint64_t counts[2] = {a.n_cus, db.dw_sep ? a.n_chroma_cus : 0};
    thread_local std::vector<CuTail> tails;
    auto fits8 = [](int32_t v) { return v >= -127 && v <= 127; };
    for (int l = 0; l < (db.dw_sep ? 2 : 1); ++l) {
      // compact heads when every CU of the list fits them (QPs and sub-block counts in 8 bits)
      bool compact = true;
      for (uint64_t i = 0; i < counts[l] && compact; ++i) {
        const h266_deblock_cu &c = lists[l][i];
        const bool legacy = c.qp_c[0] == INT32_MIN;
        compact = fits8(c.qp_y) && (legacy || (fits8(c.qp_c[0]) && fits8(c.qp_c[1]) && fits8(c.qp_c[2]))) &&
                  c.num_sb_x <= 255 && c.num_sb_y <= 255 && c.x + c.w <= 65535 && c.y + c.h <= 65535;
      }
      w.compact[l] = compact;
      const size_t hb = compact ? sizeof(CuCompact) : kCuHeadBytes;
      size_t off;
      uint8_t *heads = blob.alloc(counts[l] * hb, off);
      (l ? pr.st.dw_ccus : pr.st.dw_cus) = off;
      tails.clear();
      for (uint64_t i = 0; i < counts[l]; ++i) {
        const h266_deblock_cu &c = lists[l][i];
        if (compact) {
          CuCompact k;
          k.x = (uint16_t)c.x;
          k.y = (uint16_t)c.y;
          k.w = (uint16_t)c.w;
          k.h = (uint16_t)c.h;
          const bool legacy = c.qp_c[0] == INT32_MIN;
          k.qp_y = (int8_t)c.qp_y;
          k.qp_c[0] = legacy ? (int8_t)-128 : (int8_t)c.qp_c[0];
          k.qp_c[1] = legacy ? (int8_t)0 : (int8_t)c.qp_c[1];
          k.qp_c[2] = legacy ? (int8_t)0 : (int8_t)c.qp_c[2];
          const uint8_t fl[13] = {c.intra,        c.tu_y_coded, c.tu_cb_coded, c.tu_cr_coded, c.bdpcm_luma,
                                  c.bdpcm_chroma, c.plt,        c.joint_cbcr2, c.ciip,        c.ibc,
                                  c.has_num_sb,   c.has_tu64,   c.has_tb_split};
          k.flags = 0;
          for (int b = 0; b < 13; ++b) k.flags |= (uint16_t)((fl[b] != 0) << b);
          k.nsb_x = (uint8_t)c.num_sb_x;
          k.nsb_y = (uint8_t)c.num_sb_y;
          std::memcpy(heads + i * sizeof(CuCompact), &k, sizeof k);
        } else {
          std::memcpy(heads + i * kCuHeadBytes, &c, kCuHeadBytes);
        }
        // only sub-block grids, TB splits and 64-sample TU tiling put edges inside a CU
        if (c.has_num_sb || c.has_tb_split || (c.has_tu64 && std::max(c.w, c.h) > 64))
          w.max_cu_dim = std::max(w.max_cu_dim, std::max(c.w, c.h));
        if (c.has_tu64 || c.has_tb_split) {
          CuTail t;
          t.index = (uint32_t)i;
          std::memcpy(t.tail, reinterpret_cast<const uint8_t *>(&c) + kCuHeadBytes, sizeof t.tail);
          tails.push_back(t);
        }
      }
      w.n_tails[l] = tails.size();
      pr.st.dw_tails[l] = blob.put(tails.data(), tails.size() * sizeof(CuTail));
    }
    if (db.dw_mv) {
      // Motion by CU when the grid covers the picture and every luma CU's
      // cells agree (the walk reads motion only inside CUs): one record per
      // CU instead of one per 4x4 cell.
      const h266_deblock_mv_grid &g = *a.mv_grid;
      bool per_cu = g.cells_w >= (uint64_t)(w.w + 3) / 4 && g.cells_h >= (uint64_t)(w.h + 3) / 4;
      // Intra CUs read no motion (bS 2 comes first), so only the others' records travel.
      thread_local std::vector<CuMotionRec> rec;
      rec.clear();
      for (uint64_t i = 0; i < a.n_cus && per_cu; ++i) {
        const h266_deblock_cu &c = a.cus[i];
        if (c.intra) continue;
        const h266_deblock_mv_cell *first = &g.cells[(c.y / 4) * g.cells_w + c.x / 4];
        const size_t w4 = c.w / 4;
        // every cell of the first row equals its left neighbour, every row the first
        per_cu = w4 < 2 || std::memcmp(first + 1, first, (w4 - 1) * sizeof *first) == 0;
        for (uint32_t y = c.y / 4 + 1; y < (c.y + c.h) / 4 && per_cu; ++y)
          per_cu = std::memcmp(&g.cells[y * g.cells_w + c.x / 4], first, w4 * sizeof *first) == 0;
        CuMotionRec r;
        r.index = (uint32_t)i;
        r.m = *first;
        rec.push_back(r);
      }
      db.dw_mv_cu = per_cu;
      w.mv_by_cu = per_cu;
      w.n_mv_recs = per_cu ? rec.size() : 0;
      if (per_cu) pr.st.dw_mv = blob.put(rec.data(), rec.size() * sizeof(CuMotionRec));
      else pr.st.dw_mv = blob.put(a.mv_grid->cells, w.mv_w * w.mv_h * sizeof(h266_deblock_mv_cell));
    }
    pr.st.dw_cols = blob.put(a.no_filter_cols, a.n_no_filter_cols * sizeof(uint32_t));
    pr.st.dw_rows = blob.put(a.no_filter_rows, a.n_no_filter_rows * sizeof(uint32_t));
  } else {
    H266_TRY(build_deblock_plan(pic, a.cus, a.n_cus, a.chroma_cus, a.n_chroma_cus, a.mv_grid, a.deblock,
                                a.chroma_format_idc, a.no_filter_cols, a.n_no_filter_cols, a.no_filter_rows,
                                a.n_no_filter_rows, pr.plan, pool));
    stage_deblock(pr.plan, pr.blob, pr.st, pr.db);
  }
  if (pr.h.do_sao || pr.h.do_alf) stage_pass2(pr.h, pr.blob, pr.st);
  return H266_OK;
}

// The device walk's inputs rebased onto the uploaded blob at `base`.
DeviceWalkIn device_walk_in(const uint8_t *base, const Staged &st, const DbSide &db) {
  DeviceWalkIn in = db.dw;
  in.heads[0] = base + st.dw_cus;
  in.heads[1] = db.dw_sep ? base + st.dw_ccus : in.heads[0];
  if (!db.dw_sep) in.compact[1] = in.compact[0];
  for (int l = 0; l < 2; ++l) in.tails[l] = reinterpret_cast<const CuTail *>(base + st.dw_tails[db.dw_sep ? l : 0]);
  if (!db.dw_sep) in.n_tails[1] = in.n_tails[0];
  in.mv_cells = db.dw_mv && !db.dw_mv_cu ? reinterpret_cast<const h266_deblock_mv_cell *>(base + st.dw_mv) : nullptr;
  in.mv_recs = db.dw_mv && db.dw_mv_cu ? reinterpret_cast<const CuMotionRec *>(base + st.dw_mv) : nullptr;
  in.mv_by_cu = db.dw_mv && db.dw_mv_cu;
  in.nf_cols = reinterpret_cast<const uint32_t *>(base + st.dw_cols);
  in.nf_rows = reinterpret_cast<const uint32_t *>(base + st.dw_rows);
  return in;
}

// Launches the chain: LMCS (LUT already built) -> deblock -> SAO/ALF.  With a
// pass 2 the deblocked planes go to the scratch planes S, else in place.
int exec_chain(h266_ctx *ctx, cudaStream_t stream, const uint8_t *base, const Staged &st, const DbSide &db,
               const Pass2Host &h, const uint16_t *lut, int dbd, const DPlane P[3], const DPlane S[3],
               uint8_t *walk = nullptr) {
  if (!h.do_sao && !h.do_alf) return run_deblock(ctx, stream, base, st, db, P, P, lut, dbd, walk);
  H266_TRY(run_deblock(ctx, stream, base, st, db, P, S, lut, dbd, walk));
  return run_pass2(ctx, stream, h.args, h.do_sao, h.do_alf, h.packed, base, st, S, P);
}

// Queues the chain for one prepared picture whose planes are the device
// views `P` on lane `ln`.
int issue_chain(h266_ctx *ctx, Lane &ln, Prep &pr, const DPlane P[3], const h266_in_loop_filter_args &a) {
  ctx->h2d_bytes += pr.blob.size();
  if (pr.staged_pinned) {  // staged by the worker: copy straight from its pinned buffer
    H266_TRY(ln.side.ensure(pr.blob.size()));
    H266_CUDA(cudaMemcpyAsync(ln.side.ptr, pr.pinned.ptr, pr.blob.size(), cudaMemcpyHostToDevice, ln.stream));
    H266_CUDA(cudaEventRecord(pr.uploaded, ln.stream));
    pr.st.base = ln.side.as<uint8_t>();
  } else {
    H266_TRY(upload_blob(ln, pr.blob, &pr.st.base));
  }
  const uint16_t *lut = nullptr;
  if (a.lmcs) {
    H266_TRY(ln.lut.ensure(65536 * 2));
    H266_TRY(build_lut(ctx, ln.stream, ln.lut.as<uint16_t>(), *a.lmcs, a.lmcs_min_bin_idx, a.lmcs_max_bin_idx));
    lut = ln.lut.as<uint16_t>();
  }
  DPlane S[3];
  if (pr.h.do_sao || pr.h.do_alf) H266_TRY(ensure_scratch(ln, P, S));
  uint8_t *walk = nullptr;
  if (pr.db.device_walk) {
    H266_TRY(ln.walk.ensure(device_walk_bytes(pr.db.dw)));
    walk = ln.walk.as<uint8_t>();
  }
  return exec_chain(ctx, ln.stream, pr.st.base, pr.st, pr.db, pr.h, lut, (int)a.deblock.bit_depth, P, S, walk);
}

// Device-built side information unless a cross-check switch selects another path.
bool device_sideinfo_allowed(const h266_ctx *ctx) {
  return !ctx->force_host_sideinfo && !ctx->force_global_deblock && !ctx->force_strip_deblock;
}

// Worker pool of the context (created on first use): as many threads as the
// host offers, at most 16.
// The context's preparation workers: the "prep_threads" tuning, else half the
// host threads less two (2..16).  More workers prepare faster but slow the
// issuing thread's copies and launches (measured on a 16-thread host: 6
// workers gave the shortest end-to-end batch).
TaskPool *ctx_pool(h266_ctx *ctx) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned want = ctx->tuning.prep_threads > 0 ? (unsigned)ctx->tuning.prep_threads
                                                     : std::max(2u, std::min(hw / 2 > 2 ? hw / 2 - 2 : 2u, 16u));
  if (!ctx->pool || ctx->pool->size() != want) ctx->pool.reset(new TaskPool(want));
  return ctx->pool.get();
}

Prep &ctx_prep(h266_ctx *ctx, size_t i) {
  while (ctx->preps.size() <= i) ctx->preps.emplace_back(new Prep());
  return *ctx->preps[i];
}

// The chain for one picture whose planes are already device views `P`, on the
// main lane; its deblocking plan is built with the worker pool.
int chain_on_device(h266_ctx *ctx, const h266_picture &pic, const DPlane P[3], const h266_in_loop_filter_args &a) {
  Prep &pr = ctx_prep(ctx, 0);
  H266_TRY(prepare_chain(pr, pic, a, ctx_pool(ctx), device_sideinfo_allowed(ctx)));
  return issue_chain(ctx, ctx->main, pr, P, a);
}

bool same_geometry(const h266_picture &a, const h266_picture &b) {
  const h266_plane *x[3] = {&a.luma, &a.cb, &a.cr}, *y[3] = {&b.luma, &b.cb, &b.cr};
  for (int i = 0; i < 3; ++i)
    if (x[i]->width != y[i]->width || x[i]->height != y[i]->height || x[i]->bit_depth != y[i]->bit_depth) return false;
  return true;
}

}  // namespace

// ======================================================================= C ABI
// ---------------------------------------------------------------- recon-side LMCS, output dump
namespace {

// Samples of a plane already covered by the rectangles of the current launch
// group: a rectangle meeting one of them starts the next group, so every
// launch works on disjoint rectangles and groups run in list order.
// Cells are g x g samples, g the coarsest grid every rectangle edge lies on
// (CU and TB edges: 4 luma / 2 chroma), so the test stays exact.
// One bit per cell of a grid of 2^sh x 2^sh samples over a plane: the
// rectangles one launch may take in any order are those whose cells are all
// still clear.
struct Coverage {
  uint32_t wpr = 0, sh = 0;
  std::vector<uint64_t> bits;
  void reset(uint32_t w, uint32_t h, uint32_t sh_) {
    sh = sh_;
    const uint32_t g = 1u << sh;
    wpr = (((w + g - 1) >> sh) + 63) / 64;
    bits.assign((size_t)wpr * ((h + g - 1) >> sh), 0);
  }
  void clear() { std::fill(bits.begin(), bits.end(), 0); }
  // Marks the rectangle's cells and returns true; returns false, marking
  // nothing, when one of them is marked already.
  bool claim(uint32_t x, uint32_t y, uint32_t rw, uint32_t rh) {
    const uint32_t g = 1u << sh;
    const uint32_t cx = x >> sh, cw = (rw + g - 1) >> sh, ch = (rh + g - 1) >> sh;
    const uint32_t w0 = cx >> 6, w1 = (cx + cw - 1) >> 6;
    uint64_t *row = bits.data() + (size_t)(y >> sh) * wpr;
    auto mask = [&](uint32_t wi) {
      const uint32_t lo = std::max(cx, wi * 64) - wi * 64, hi = std::min(cx + cw, wi * 64 + 64) - wi * 64;
      return hi - lo == 64 ? ~0ull : (((1ull << (hi - lo)) - 1) << lo);
    };
    if (w0 == w1) {  // the common case: one word per row
      const uint64_t m = mask(w0);
      uint64_t hit = 0;
      for (uint32_t r = 0; r < ch; ++r) hit |= row[(size_t)r * wpr + w0] & m;
      if (hit) return false;
      for (uint32_t r = 0; r < ch; ++r) row[(size_t)r * wpr + w0] |= m;
      return true;
    }
    for (uint32_t r = 0; r < ch; ++r)
      for (uint32_t wi = w0; wi <= w1; ++wi)
        if (row[(size_t)r * wpr + wi] & mask(wi)) return false;
    for (uint32_t r = 0; r < ch; ++r)
      for (uint32_t wi = w0; wi <= w1; ++wi) row[(size_t)r * wpr + wi] |= mask(wi);
    return true;
  }
};

// log2 of the coarsest of 4, 2, 1 dividing every value folded into `acc` (an OR).
uint32_t grid_shift(uint32_t acc) { return (acc & 3) == 0 ? 2 : ((acc & 1) == 0 ? 1 : 0); }

constexpr uint32_t kPieceSamples = 1024;  // residual-add piece
constexpr uint32_t kPieceCells = 1024;    // forward-map count piece

h266_picture plane_view(const h266_picture &pic, int keep) {  // the picture with only plane `keep` (-1: chroma)
  h266_picture v = pic;
  h266_plane *pl[3] = {&v.luma, &v.cb, &v.cr};
  for (int i = 0; i < 3; ++i)
    if (keep >= 0 ? i != keep : i == 0) pl[i]->width = pl[i]->height = 0;
  return v;
}

int sync_read(Lane &ln, void *host, const void *dev, size_t n) {
  H266_CUDA(cudaMemcpyAsync(host, dev, n, cudaMemcpyDeviceToHost, ln.stream));
  H266_CUDA(cudaStreamSynchronize(ln.stream));
  return H266_OK;
}

}  // namespace

extern "C" {

const char *h266_last_error(void) { return g_last_error.c_str(); }

int h266_ctx_create(int device, h266_ctx **out) {
  if (!out) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL out");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return set_error(H266_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= n) return set_error(H266_ERR_NO_DEVICE, "device ordinal out of range");
  Guard g(device);
  h266_ctx *c = new h266_ctx();
  c->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return cuda_error(e, "h266_ctx_create");
  }
  c->stream = c->own;
  const int rc = c->main.init(c->own);
  if (rc != H266_OK) {
    c->main.release();
    cudaStreamDestroy(c->own);
    delete c;
    return rc;
  }
  const char *fs = std::getenv("H266_FORCE_SCALAR_ALF");
  c->force_scalar = fs && fs[0] == '1';
  const char *fg = std::getenv("H266_FORCE_GLOBAL_DEBLOCK");
  c->force_global_deblock = fg && fg[0] == '1';
  const char *fstrip = std::getenv("H266_FORCE_STRIP_DEBLOCK");
  c->force_strip_deblock = fstrip && fstrip[0] == '1';
  const char *fhost = std::getenv("H266_FORCE_HOST_SIDEINFO");
  c->force_host_sideinfo = fhost && fhost[0] == '1';
  *out = c;
  return H266_OK;
}

int h266_ctx_destroy(h266_ctx *ctx) {
  if (!ctx) return H266_OK;
  Guard g(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto &l : ctx->lanes) {
    cudaStreamSynchronize(l->stream);
    l->release();
  }
  for (auto &l : ctx->glanes) l->release();
  for (cudaStream_t st : {ctx->e2e_up, ctx->e2e_down})
    if (st) cudaStreamSynchronize(st), cudaStreamDestroy(st);
  ctx->main.release();
  ctx->pool.reset();
  for (auto &e : ctx->ev_pool) cudaEventDestroy(e);
  for (auto &e : ctx->ev_pending) {
    cudaEventDestroy(e.second.first);
    cudaEventDestroy(e.second.second);
  }
  ctx->batch.release();
  if (ctx->own) cudaStreamDestroy(ctx->own);
  delete ctx;
  return H266_OK;
}

int h266_ctx_set_stream(h266_ctx *ctx, void *stream) {
  H266_TRY(check_ctx(ctx));
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own;
  ctx->main.stream = ctx->stream;
  return H266_OK;
}

int h266_ctx_synchronize(h266_ctx *ctx) {
  H266_TRY(check_ctx(ctx));
  Guard g(ctx->device);
  H266_CUDA(cudaStreamSynchronize(ctx->stream));
  uint32_t timeouts = 0, db_timeouts = 0;
  H266_TRY(pass2_wait_timeouts(&timeouts));
  H266_TRY(deblock_wait_timeouts(&db_timeouts));
  if (timeouts)
    return set_error(H266_ERR_TIMEOUT, std::to_string(timeouts) +
                                           " SAO/ALF tiles gave up waiting for their window copies (left unfiltered)");
  if (db_timeouts)
    return set_error(H266_ERR_TIMEOUT, std::to_string(db_timeouts) +
                                           " deblocking tiles gave up waiting for their region copies (left unwritten)");
  return H266_OK;
}

uint64_t h266_ctx_kernel_launches(const h266_ctx *ctx) { return ctx ? ctx->launches : 0; }

int h266_ctx_transfer_bytes(const h266_ctx *ctx, uint64_t *h2d, uint64_t *d2h) {
  H266_TRY(check_ctx(const_cast<h266_ctx *>(ctx)));
  if (h2d) *h2d = ctx->h2d_bytes;
  if (d2h) *d2h = ctx->d2h_bytes;
  return H266_OK;
}

int h266_derive_lmcs(const h266_lmcs_data *data, uint32_t bit_depth, h266_lmcs_derived *out) {
  return derive_lmcs(data, bit_depth, out);
}

int h266_lmcs_inverse_map_luma(h266_ctx *ctx, h266_picture *pic, const h266_lmcs_derived *lmcs, uint32_t mn,
                               uint32_t mx) {
  H266_TRY(check_ctx(ctx));
  H266_TRY(check_picture(pic));
  if (!lmcs) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL lmcs");
  H266_TRY(check_lmcs(lmcs, mn, mx));
  Guard g(ctx->device);
  Lane &ln = ctx->main;
  DPlane P[3];
  H266_TRY(picture_to_device(ln, *pic, P));
  H266_TRY(ln.lut.ensure(65536 * 2));
  H266_TRY(build_lut(ctx, ln.stream, ln.lut.as<uint16_t>(), *lmcs, mn, mx));
  H266_TRY(plane_map(ctx, ln.stream, P[0], P[0], ln.lut.as<uint16_t>()));
  return picture_from_device(ln, *pic);
}

int h266_apply_deblocking_clipped(h266_ctx *ctx, h266_picture *pic, const h266_deblock_cu *cus, uint64_t n_cus,
                                  const h266_deblock_cu *chroma_cus, uint64_t n_chroma_cus,
                                  const h266_deblock_mv_grid *mv_grid, const h266_deblock_params *params,
                                  uint32_t cfi, const uint32_t *nf_cols, uint64_t n_cols, const uint32_t *nf_rows,
                                  uint64_t n_rows) {
  H266_TRY(check_ctx(ctx));
  H266_TRY(check_picture(pic));
  if (!params) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL params");
  if ((n_cus && !cus) || (n_cols && !nf_cols) || (n_rows && !nf_rows))
    return set_error(H266_ERR_INVALID_ARGUMENT, "NULL list with nonzero length");
  Guard g(ctx->device);
  Prep &pr = ctx_prep(ctx, 0);
  H266_TRY(build_deblock_plan(*pic, cus, n_cus, chroma_cus, n_chroma_cus, mv_grid, *params, cfi, nf_cols, n_cols,
                              nf_rows, n_rows, pr.plan, ctx_pool(ctx)));
  Lane &ln = ctx->main;
  DPlane P[3];
  H266_TRY(picture_to_device(ln, *pic, P));
  Staged st;
  DbSide db;
  pr.blob.clear();
  stage_deblock(pr.plan, pr.blob, st, db);
  H266_TRY(upload_blob(ln, pr.blob, &st.base));
  H266_TRY(run_deblock(ctx, ln.stream, st.base, st, db, P, P, nullptr, (int)params->bit_depth));
  return picture_from_device(ln, *pic);
}

static int pass2_entry(h266_ctx *ctx, h266_picture *pic, const Pass2Inputs &in) {
  H266_TRY(check_ctx(ctx));
  H266_TRY(check_picture(pic));
  if (in.cols && !in.rows) return set_error(H266_ERR_INVALID_ARGUMENT, "row bounds NULL while col bounds are not");
  Guard g(ctx->device);
  Prep &pr = ctx_prep(ctx, 0);
  Pass2Host &h = pr.h;
  H266_TRY(build_pass2(*pic, in, h));
  Lane &ln = ctx->main;
  DPlane P[3];
  H266_TRY(picture_to_device(ln, *pic, P));
  if (h.do_sao || h.do_alf) {
    Staged st;
    pr.blob.clear();
    stage_pass2(h, pr.blob, st);
    H266_TRY(upload_blob(ln, pr.blob, &st.base));
    DPlane S[3];
    H266_TRY(ensure_scratch(ln, P, S));
    for (int i = 0; i < 3; ++i) H266_TRY(plane_map(ctx, ln.stream, S[i], P[i], nullptr));
    H266_TRY(run_pass2(ctx, ln.stream, h.args, h.do_sao, h.do_alf, h.packed, st.base, st, S, P));
  }
  return picture_from_device(ln, *pic);
}

int h266_apply_sao_clipped(h266_ctx *ctx, h266_picture *pic, const h266_sao_picture *sao_pic,
                           const h266_sao_config *cfg, const uint32_t *col_bd, uint64_t n_col, const uint32_t *row_bd,
                           uint64_t n_row) {
  if (!sao_pic || !cfg) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL SAO picture / config");
  Pass2Inputs in;
  in.sao = sao_pic;
  in.sao_cfg = cfg;
  in.cols = col_bd;
  in.rows = row_bd;
  in.n_cols = n_col;
  in.n_rows = n_row;
  return pass2_entry(ctx, pic, in);
}

int h266_apply_alf_clipped(h266_ctx *ctx, h266_picture *pic, const h266_alf_picture *alf_pic,
                           const h266_alf_config *cfg, const h266_alf_aps_binding *binding, const uint32_t *col_bd,
                           uint64_t n_col, const uint32_t *row_bd, uint64_t n_row) {
  if (!alf_pic || !cfg) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL ALF picture / config");
  Pass2Inputs in;
  in.alf = alf_pic;
  in.alf_cfg = cfg;
  in.binding = binding;
  in.cols = col_bd;
  in.rows = row_bd;
  in.n_cols = n_col;
  in.n_rows = n_row;
  return pass2_entry(ctx, pic, in);
}

// The chroma ALF (cc = false) and CC-ALF (cc = true) decisions: one chain
// SAO/ALF pass per candidate into its own chroma plane (the other chroma
// plane left out, luma written to a throw-away plane), per-CTB SSE, pick,
// commit.
static int chroma_trials(h266_ctx *ctx, const h266_picture *src, h266_picture *rec, const uint16_t *pre_luma,
                         h266_alf_ctb *apply, uint64_t n_apply, const h266_alf_aps_data *aps, uint32_t comp, bool cc,
                         uint32_t log2, uint32_t bd, uint32_t cfi, const uint32_t *col_bd, uint64_t n_col,
                         const uint32_t *row_bd, uint64_t n_row) {
  H266_TRY(check_ctx(ctx));
  H266_TRY(check_picture(src));
  H266_TRY(check_picture(rec));
  if (!apply || !aps) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL apply_pic / aps");
  if (comp != 1 && comp != 2) return set_error(H266_ERR_INVALID_ARGUMENT, "component must be 1 (Cb) or 2 (Cr)");
  if (cc && !pre_luma) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL pre_luma_alf");
  if (col_bd && !row_bd) return set_error(H266_ERR_INVALID_ARGUMENT, "row bounds NULL while col bounds are not");
  if (cfi > 3) return set_error(H266_ERR_INVALID_ARGUMENT, "chroma_format_idc must be 0..3");
  if (cfi == 0) return H266_OK;  // monochrome (src/alf_enc.rs:639-641, 946-948)
  uint32_t n_cand;
  if (!cc) {
    if (!aps->alf_chroma_filter_signal_flag) return H266_OK;  // src/alf_enc.rs:642-648
    n_cand = aps->n_chroma_filters;
    if (n_cand > 8) return set_error(H266_ERR_INVALID_ARGUMENT, "chroma APS: more than 8 filters");
  } else {
    n_cand = comp == 1 ? aps->n_cc_cb_filters : aps->n_cc_cr_filters;  // src/alf_enc.rs:949-955
    if (n_cand > 4) return set_error(H266_ERR_INVALID_ARGUMENT, "CC-ALF: more than 4 filters");
  }
  if (n_cand == 0) return H266_OK;
  if (cfi != 1) return set_error(H266_ERR_UNSUPPORTED, "chroma ALF trials need 4:2:0");
  if (bd < 8 || bd > 14) return set_error(H266_ERR_UNSUPPORTED, "chroma ALF trials need BitDepth 8..14");
  if (log2 < 5 || log2 > 7) return set_error(H266_ERR_UNSUPPORTED, "chroma ALF trials need CtbLog2SizeY in 5..7");
  const uint32_t ctb = 1u << log2;
  const uint32_t wc = (rec->luma.width + ctb - 1) / ctb, hc = (rec->luma.height + ctb - 1) / ctb;
  const int n = (int)((uint64_t)wc * hc);
  if (n_apply != (uint64_t)n) return set_error(H266_ERR_GRID_MISMATCH, "apply_pic size != CTB grid of rec");
  const h266_plane &rp = comp == 1 ? rec->cb : rec->cr, &sp = comp == 1 ? src->cb : src->cr;
  if ((uint64_t)rp.width * rp.height == 0) return H266_OK;  // nothing to filter: every trial ties "off"
  Guard g(ctx->device);
  Lane &ln = ctx->main;
  Prep &pr = ctx_prep(ctx, 0);
  Pass2Host &h = pr.h;
  DPlane R[3];
  H266_TRY(picture_to_device(ln, *rec, R));
  ctx->h2d_bytes += host_plane_bytes(*rec);
  DPlane S{}, PL = R[0];
  if (src->mem == H266_MEM_DEVICE || (uint64_t)sp.width * sp.height == 0) {
    S = dplane(sp, sp.samples, (int64_t)std::max<uint64_t>(sp.stride, 1));
  } else {
    const size_t row = (size_t)sp.width * 2;
    H266_TRY(ln.scratch[1].ensure(row * sp.height));
    H266_CUDA(cudaMemcpy2DAsync(ln.scratch[1].ptr, row, sp.samples, (size_t)sp.stride * 2, row, sp.height,
                                cudaMemcpyHostToDevice, ln.stream));
    S = dplane(sp, ln.scratch[1].as<uint16_t>(), sp.width);
    ctx->h2d_bytes += row * sp.height;
  }
  if (cc) {  // the trials' luma: the samples before luma ALF, rec's luma layout
    if (rec->mem == H266_MEM_DEVICE) {
      PL = dplane(rec->luma, const_cast<uint16_t *>(pre_luma), (int64_t)rec->luma.stride);
    } else {
      const size_t row = (size_t)rec->luma.width * 2;
      H266_TRY(ln.scratch[0].ensure(row * rec->luma.height));
      H266_CUDA(cudaMemcpy2DAsync(ln.scratch[0].ptr, row, pre_luma, (size_t)rec->luma.stride * 2, row,
                                  rec->luma.height, cudaMemcpyHostToDevice, ln.stream));
      PL = dplane(rec->luma, ln.scratch[0].as<uint16_t>(), rec->luma.width);
      ctx->h2d_bytes += row * rec->luma.height;
    }
  }
  // scratch: SSE table, picks, one chroma plane per candidate, a throw-away luma plane
  const int cols = (int)n_cand + 1;
  const size_t cw = rp.width, chh = rp.height, lw = rec->luma.width, lh = rec->luma.height;
  const size_t sse_b = (size_t)n * cols * 8, pick_b = ((size_t)n + 255) & ~(size_t)255;
  const size_t plane_b = ((cw * chh * 2) + 255) & ~(size_t)255, luma_b = lw * lh * 2;
  H266_TRY(ln.walk.ensure(sse_b + pick_b + plane_b * n_cand + luma_b + 256));
  uint8_t *w = ln.walk.as<uint8_t>();
  auto *d_sse = reinterpret_cast<unsigned long long *>(w);
  auto *d_pick = reinterpret_cast<int8_t *>(w + sse_b);
  auto *d_trials = reinterpret_cast<uint16_t *>(w + sse_b + pick_b);
  auto *d_luma = reinterpret_cast<uint16_t *>(w + sse_b + pick_b + plane_b * n_cand);
  const int cwc = (int)(ctb / 2), chc = (int)(ctb / 2);
  Prof pf(ctx, ln.stream, H266_PROF_SAO_ALF);
  H266_TRY(launch_ctb_sse(ln.stream, S, R[comp], cwc, chc, (int)wc, n, d_sse, cols, 0, &ctx->launches));
  std::vector<h266_alf_ctb> trial((size_t)n);
  h266_alf_config cfg{1, comp == 1, comp == 2, comp == 1, comp == 2, bd, log2, cfi};
  h266_alf_aps_binding binding{};
  if (!cc) binding.chroma_aps = aps;
  else if (comp == 1) binding.cc_cb_aps = aps;
  else binding.cc_cr_aps = aps;
  for (uint32_t k = 0; k < n_cand; ++k) {
    for (h266_alf_ctb &c : trial) {
      c = h266_alf_ctb{};
      if (!cc) {
        (comp == 1 ? c.cb_on : c.cr_on) = 1;
        (comp == 1 ? c.cb_alt_idx : c.cr_alt_idx) = (uint8_t)k;
      } else {
        (comp == 1 ? c.cc_cb_idc : c.cc_cr_idc) = (uint8_t)(k + 1);
      }
    }
    const h266_alf_picture ap{wc, hc, trial.data()};
    Pass2Inputs in;
    in.alf = &ap;
    in.alf_cfg = &cfg;
    in.binding = &binding;
    in.cols = col_bd;
    in.rows = row_bd;
    in.n_cols = n_col;
    in.n_rows = n_row;
    H266_TRY(build_pass2(*rec, in, h));
    if (!h.packed) return set_error(H266_ERR_UNSUPPORTED, "chroma ALF trials: coefficients outside [-128, 127]");
    Staged st;
    pr.blob.clear();
    stage_pass2(h, pr.blob, st);
    H266_TRY(upload_blob(ln, pr.blob, &st.base));
    ctx->h2d_bytes += pr.blob.size();
    const DPlane none{nullptr, 1, 0, 0};
    DPlane SRC[3] = {cc ? PL : R[0], none, none}, DST[3] = {DPlane{d_luma, (int64_t)lw, (int)lw, (int)lh}, none, none};
    SRC[comp] = R[comp];
    DST[comp] = DPlane{d_trials + (size_t)k * (plane_b / 2), (int64_t)cw, (int)cw, (int)chh};
    Pass2Args a = h.args;
    bind_pass2(a, st.base, st, SRC, DST);
    H266_TRY(launch_pass2_packed(ln.stream, a, false, true, &ctx->launches));
    H266_TRY(launch_ctb_sse(ln.stream, S, DST[comp], cwc, chc, (int)wc, n, d_sse, cols, 1 + (int)k, &ctx->launches));
  }
  H266_TRY(launch_trial_pick_commit(ln.stream, d_sse, cols, n, d_pick, R[comp], d_trials, (int64_t)(plane_b / 2),
                                    (int)cw, cwc, chc, (int)wc, &ctx->launches));
  std::vector<int8_t> pick((size_t)n);
  H266_CUDA(cudaMemcpyAsync(pick.data(), d_pick, (size_t)n, cudaMemcpyDeviceToHost, ln.stream));
  h266_picture one = *rec;  // copy back only the decided plane
  h266_plane *pl[3] = {&one.luma, &one.cb, &one.cr};
  for (int i = 0; i < 3; ++i)
    if (i != (int)comp) pl[i]->width = pl[i]->height = 0;
  H266_TRY(picture_from_device(ln, one));
  if (rec->mem == H266_MEM_DEVICE) H266_CUDA(cudaStreamSynchronize(ln.stream));
  ctx->d2h_bytes += host_plane_bytes(one) + (size_t)n;
  for (int i = 0; i < n; ++i) {
    if (pick[i] < 0) continue;
    h266_alf_ctb &e = apply[i];
    if (!cc) {
      (comp == 1 ? e.cb_on : e.cr_on) = 1;
      (comp == 1 ? e.cb_alt_idx : e.cr_alt_idx) = (uint8_t)pick[i];
    } else {
      (comp == 1 ? e.cc_cb_idc : e.cc_cr_idc) = (uint8_t)(pick[i] + 1);
    }
  }
  return H266_OK;
}

int h266_chroma_alf_decide_and_apply_clipped(h266_ctx *ctx, const h266_picture *src, h266_picture *rec,
                                             h266_alf_ctb *apply_pic, uint64_t n_apply, const h266_alf_aps_data *aps,
                                             uint32_t component, uint32_t log2, uint32_t bd, uint32_t cfi,
                                             const uint32_t *col_bd, uint64_t n_col, const uint32_t *row_bd,
                                             uint64_t n_row) {
  return chroma_trials(ctx, src, rec, nullptr, apply_pic, n_apply, aps, component, false, log2, bd, cfi, col_bd, n_col,
                       row_bd, n_row);
}

int h266_cc_alf_decide_and_apply_clipped(h266_ctx *ctx, const h266_picture *src, h266_picture *rec,
                                         const uint16_t *pre_luma_alf, h266_alf_ctb *apply_pic, uint64_t n_apply,
                                         const h266_alf_aps_data *aps, uint32_t component, uint32_t log2, uint32_t bd,
                                         uint32_t cfi, const uint32_t *col_bd, uint64_t n_col, const uint32_t *row_bd,
                                         uint64_t n_row) {
  return chroma_trials(ctx, src, rec, pre_luma_alf, apply_pic, n_apply, aps, component, true, log2, bd, cfi, col_bd,
                       n_col, row_bd, n_row);
}

int h266_sao_chroma_merge(h266_ctx *ctx, const h266_picture *src, const h266_picture *pre,
                          const h266_sao_ctb_params *indep, uint32_t wc, uint32_t hc, uint32_t bd, uint32_t log2,
                          h266_sao_ctb_params *merged, uint8_t *map) {
  H266_TRY(check_ctx(ctx));
  H266_TRY(check_picture(src));
  H266_TRY(check_picture(pre));
  const uint64_t n = (uint64_t)wc * hc;
  if (n && (!indep || !merged || !map)) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL records / map");
  if (bd < 8 || bd > 16) return set_error(H266_ERR_INVALID_ARGUMENT, "bit_depth must be 8..16");
  if (log2 < 1 || log2 > 7) return set_error(H266_ERR_INVALID_ARGUMENT, "ctb_log2_size_y must be 1..7");
  if (n > (1u << 22)) return set_error(H266_ERR_UNSUPPORTED, "CTB grid too large");
  if (pre->cb.width != pre->cr.width || pre->cb.height != pre->cr.height)
    return set_error(H266_ERR_INVALID_ARGUMENT, "Cb and Cr planes differ in size");
  if (src->cb.width < pre->cb.width || src->cb.height < pre->cb.height || src->cr.width < pre->cb.width ||
      src->cr.height < pre->cb.height)
    return set_error(H266_ERR_INVALID_ARGUMENT, "original chroma planes smaller than the reconstruction's");
  if (!n) return H266_OK;
  Guard g(ctx->device);
  Lane &ln = ctx->main;
  h266_picture cv = *pre;  // chroma only
  cv.luma.width = cv.luma.height = 0;
  DPlane P[3];
  H266_TRY(picture_to_device(ln, cv, P));
  ctx->h2d_bytes += host_plane_bytes(cv);
  const h266_plane *sp[2] = {&src->cb, &src->cr};
  DPlane S[2], Q[2] = {P[1], P[2]};
  for (int i = 0; i < 2; ++i) {
    const h266_plane &p = *sp[i];
    if (src->mem == H266_MEM_DEVICE || (uint64_t)p.width * p.height == 0) {
      S[i] = dplane(p, p.samples, (int64_t)std::max<uint64_t>(p.stride, 1));
      continue;
    }
    const size_t row = (size_t)p.width * 2;
    H266_TRY(ln.scratch[1 + i].ensure(row * p.height));
    H266_CUDA(cudaMemcpy2DAsync(ln.scratch[1 + i].ptr, row, p.samples, (size_t)p.stride * 2, row, p.height,
                                cudaMemcpyHostToDevice, ln.stream));
    S[i] = dplane(p, ln.scratch[1 + i].as<uint16_t>(), p.width);
    ctx->h2d_bytes += row * p.height;
  }
  Prep &pr = ctx_prep(ctx, 0);
  pr.blob.clear();
  Blob blob{pr.blob};
  const size_t off = blob.put(indep, n * sizeof(h266_sao_ctb_params));
  uint8_t *base = nullptr;
  H266_TRY(upload_blob(ln, pr.blob, &base));
  ctx->h2d_bytes += pr.blob.size();
  const size_t rec_b = n * sizeof(h266_sao_ctb_params), map_b = (n + 255) & ~(uint64_t)255;
  H266_TRY(ln.walk.ensure(rec_b + map_b + sao_merge_work_bytes(n) + 256));
  auto *d_merged = ln.walk.as<h266_sao_ctb_params>();
  auto *d_map = ln.walk.as<uint8_t>() + rec_b;
  void *d_work = ln.walk.as<uint8_t>() + ((rec_b + map_b + 255) & ~(size_t)255);
  {
    Prof pf(ctx, ln.stream, H266_PROF_SAO_ALF);
    H266_TRY(launch_sao_chroma_merge(ln.stream, S, Q, (int)bd, (1 << log2) / 2, (int)wc, (int)hc,
                                     reinterpret_cast<const h266_sao_ctb_params *>(base + off), d_merged, d_map,
                                     d_work, &ctx->launches));
  }
  H266_CUDA(cudaMemcpyAsync(merged, d_merged, rec_b, cudaMemcpyDeviceToHost, ln.stream));
  H266_TRY(sync_read(ln, map, d_map, n));
  ctx->d2h_bytes += rec_b + n;
  return H266_OK;
}

int h266_sao_chroma_merge_batch(h266_ctx *ctx, uint32_t np, const h266_picture *const *srcs,
                                const h266_picture *const *pres, const h266_sao_ctb_params *const *indeps,
                                const uint32_t *wcs, const uint32_t *hcs, uint32_t bd, uint32_t log2,
                                h266_sao_ctb_params *const *merged, uint8_t *const *maps) {
  H266_TRY(check_ctx(ctx));
  if (np && (!srcs || !pres || !indeps || !wcs || !hcs || !merged || !maps))
    return set_error(H266_ERR_INVALID_ARGUMENT, "NULL batch arrays");
  if (bd < 8 || bd > 16) return set_error(H266_ERR_INVALID_ARGUMENT, "bit_depth must be 8..16");
  if (log2 < 1 || log2 > 7) return set_error(H266_ERR_INVALID_ARGUMENT, "ctb_log2_size_y must be 1..7");
  // layout of the device work area: per picture its merged records, map and work, 256-byte sections
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  std::vector<size_t> off_rec(np), off_map(np), off_work(np);
  size_t total = 0;
  uint32_t n_diags = 0;
  for (uint32_t i = 0; i < np; ++i) {
    const h266_picture *src = srcs[i], *pre = pres[i];
    H266_TRY(check_picture(src));
    H266_TRY(check_picture(pre));
    if (src->mem != H266_MEM_DEVICE || pre->mem != H266_MEM_DEVICE)
      return set_error(H266_ERR_INVALID_ARGUMENT, "the batched merge takes device pictures (H266_MEM_DEVICE)");
    const uint64_t n = (uint64_t)wcs[i] * hcs[i];
    if (n && (!indeps[i] || !merged[i] || !maps[i])) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL records / map");
    if (n > (1u << 22)) return set_error(H266_ERR_UNSUPPORTED, "CTB grid too large");
    if (pre->cb.width != pre->cr.width || pre->cb.height != pre->cr.height)
      return set_error(H266_ERR_INVALID_ARGUMENT, "Cb and Cr planes differ in size");
    if (src->cb.width < pre->cb.width || src->cb.height < pre->cb.height || src->cr.width < pre->cb.width ||
        src->cr.height < pre->cb.height)
      return set_error(H266_ERR_INVALID_ARGUMENT, "original chroma planes smaller than the reconstruction's");
    off_rec[i] = total;
    total += al(n * sizeof(h266_sao_ctb_params));
    off_map[i] = total;
    total += al(n);
    off_work[i] = total;
    total += al(sao_merge_work_bytes(n));
    if (n) n_diags = std::max(n_diags, wcs[i] + hcs[i] - 1);
  }
  if (!np || !n_diags) return H266_OK;
  Guard g(ctx->device);
  Lane &ln = ctx->main;
  H266_TRY(ln.walk.ensure(std::max<size_t>(total, 256)));
  uint8_t *work = ln.walk.as<uint8_t>();
  H266_CUDA(cudaMemsetAsync(work, 0, total, ln.stream));  // per-CTB arrival counts start at zero
  // one upload: every picture's independent records, merge parameters and per-diagonal picture tables
  Prep &pr = ctx_prep(ctx, 0);
  pr.blob.clear();
  Blob blob{pr.blob};
  std::vector<size_t> off_ind(np);
  for (uint32_t i = 0; i < np; ++i)
    off_ind[i] = blob.put(indeps[i], (size_t)wcs[i] * hcs[i] * sizeof(h266_sao_ctb_params));
  std::vector<uint32_t> first((size_t)n_diags * (np + 1), 0), totals(n_diags, 0);
  for (uint32_t d = 0; d < n_diags; ++d)
    for (uint32_t i = 0; i < np; ++i) {
      const int wc = (int)wcs[i], hc = (int)hcs[i];
      int c = 0;
      if (wc && hc && (int)d <= wc + hc - 2) c = std::min(hc - 1, (int)d) - std::max(0, (int)d - (wc - 1)) + 1;
      first[(size_t)d * (np + 1) + i + 1] = first[(size_t)d * (np + 1) + i] + (uint32_t)std::max(c, 0);
      totals[d] = first[(size_t)d * (np + 1) + i + 1];
    }
  const size_t off_first = blob.put(first.data(), first.size() * sizeof(uint32_t));
  const size_t asz = sao_merge_args_size();
  std::vector<uint8_t> args(asz * np);
  const size_t off_args = blob.put(args.data(), args.size());  // filled in below, once the base is known
  uint8_t *base = nullptr;
  H266_TRY(ln.side.ensure(pr.blob.size()));
  base = ln.side.as<uint8_t>();
  for (uint32_t i = 0; i < np; ++i) {
    const h266_picture &src = *srcs[i], &pre = *pres[i];
    const DPlane S[2] = {dplane(src.cb, src.cb.samples, (int64_t)std::max<uint64_t>(src.cb.stride, 1)),
                         dplane(src.cr, src.cr.samples, (int64_t)std::max<uint64_t>(src.cr.stride, 1))};
    const DPlane Q[2] = {dplane(pre.cb, pre.cb.samples, (int64_t)std::max<uint64_t>(pre.cb.stride, 1)),
                         dplane(pre.cr, pre.cr.samples, (int64_t)std::max<uint64_t>(pre.cr.stride, 1))};
    fill_sao_merge_args(pr.blob.data() + off_args + asz * i, S, Q, (int)bd, (1 << log2) / 2, (int)wcs[i], (int)hcs[i],
                        reinterpret_cast<const h266_sao_ctb_params *>(base + off_ind[i]),
                        reinterpret_cast<h266_sao_ctb_params *>(work + off_rec[i]), work + off_map[i],
                        work + off_work[i]);
  }
  H266_TRY(upload_blob(ln, pr.blob, &base));
  ctx->h2d_bytes += pr.blob.size();
  {
    Prof pf(ctx, ln.stream, H266_PROF_SAO_ALF);
    H266_TRY(launch_sao_chroma_merge_batch(ln.stream, base + off_args, reinterpret_cast<const uint32_t *>(base + off_first),
                                           (int)np, (int)n_diags, totals.data(), &ctx->launches));
  }
  for (uint32_t i = 0; i < np; ++i) {
    const size_t n = (size_t)wcs[i] * hcs[i];
    if (!n) continue;
    H266_CUDA(cudaMemcpyAsync(merged[i], work + off_rec[i], n * sizeof(h266_sao_ctb_params), cudaMemcpyDeviceToHost,
                              ln.stream));
    H266_CUDA(cudaMemcpyAsync(maps[i], work + off_map[i], n, cudaMemcpyDeviceToHost, ln.stream));
    ctx->d2h_bytes += n * (sizeof(h266_sao_ctb_params) + 1);
  }
  H266_CUDA(cudaStreamSynchronize(ln.stream));
  return H266_OK;
}

int h266_sao_decide_picture(h266_ctx *ctx, const h266_picture *src, const h266_picture *rec, uint32_t log2,
                            uint32_t bd, uint32_t sao_luma, uint32_t sao_chroma, h266_sao_ctb_params *out,
                            uint64_t n_out) {
  H266_TRY(check_ctx(ctx));
  H266_TRY(check_picture(src));
  H266_TRY(check_picture(rec));
  if (!out) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL out");
  if (bd < 8 || bd > 16) return set_error(H266_ERR_INVALID_ARGUMENT, "bit_depth must be 8..16");
  if (log2 < 4 || log2 > 7) return set_error(H266_ERR_UNSUPPORTED, "CtbLog2SizeY must be 4..7");
  const uint32_t ctb = 1u << log2;
  const uint32_t wc = (rec->luma.width + ctb - 1) / ctb, hc = (rec->luma.height + ctb - 1) / ctb;
  const uint64_t n = (uint64_t)wc * hc;
  if (n_out != n) return set_error(H266_ERR_GRID_MISMATCH, "out size != CTB grid of rec");
  if (n > (1u << 22)) return set_error(H266_ERR_UNSUPPORTED, "CTB grid too large");
  Guard g(ctx->device);
  Lane &ln = ctx->main;
  DPlane R[3], S[3];
  H266_TRY(picture_to_device(ln, *rec, R));
  ctx->h2d_bytes += host_plane_bytes(*rec);
  const h266_plane *sp[3] = {&src->luma, &src->cb, &src->cr};
  for (int i = 0; i < 3; ++i) {  // the original: caller memory or a copy in the lane's scratch planes
    const h266_plane &p = *sp[i];
    if (src->mem == H266_MEM_DEVICE || (uint64_t)p.width * p.height == 0) {
      S[i] = dplane(p, p.samples, (int64_t)std::max<uint64_t>(p.stride, 1));
      continue;
    }
    const size_t row = (size_t)p.width * 2;
    H266_TRY(ln.scratch[i].ensure(row * p.height));
    H266_CUDA(cudaMemcpy2DAsync(ln.scratch[i].ptr, row, p.samples, (size_t)p.stride * 2, row, p.height,
                                cudaMemcpyHostToDevice, ln.stream));
    S[i] = dplane(p, ln.scratch[i].as<uint16_t>(), p.width);
    ctx->h2d_bytes += row * p.height;
  }
  const size_t st_bytes = sao_stats_bytes((int)n), out_bytes = n * sizeof(h266_sao_ctb_params);
  H266_TRY(ln.walk.ensure(st_bytes + out_bytes + 256));
  uint8_t *w = ln.walk.as<uint8_t>();
  auto *d_out = reinterpret_cast<h266_sao_ctb_params *>(w + st_bytes);
  auto *d_err = reinterpret_cast<uint32_t *>(w + st_bytes + ((out_bytes + 15) & ~(size_t)15));
  H266_CUDA(cudaMemsetAsync(d_err, 0, 4, ln.stream));
  {
    Prof pf(ctx, ln.stream, H266_PROF_SAO_ALF);
    H266_TRY(launch_sao_decide(ln.stream, S, R, (int)bd, (int)log2, (int)wc, (int)hc, sao_luma != 0, sao_chroma != 0,
                               w, d_err, d_out, &ctx->launches));
  }
  uint32_t err = 0;
  H266_CUDA(cudaMemcpyAsync(out, d_out, out_bytes, cudaMemcpyDeviceToHost, ln.stream));
  H266_TRY(sync_read(ln, &err, d_err, 4));
  ctx->d2h_bytes += out_bytes;
  if (err) return set_error(H266_ERR_INVALID_ARGUMENT, "SAO decision: a sample above (1 << bit_depth) - 1 has no band");
  return H266_OK;
}

int h266_lmcs_forward_map_luma_rects(h266_ctx *ctx, h266_picture *pic, const h266_lmcs_derived *lmcs,
                                     const h266_rect *rects, uint64_t n) {
  H266_TRY(check_ctx(ctx));
  H266_TRY(check_picture(pic));
  if (!lmcs) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL lmcs");
  H266_TRY(check_lmcs(lmcs, 0, 0));
  if (n && !rects) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL rects with nonzero length");
  if (n > (1ull << 28)) return set_error(H266_ERR_UNSUPPORTED, "too many rectangles");
  const uint32_t W = pic->luma.width, H = pic->luma.height;
  // Rectangles clipped as src/ctu.rs:1718-1719; the grid is the coarsest that
  // every clipped edge lies on, the span box their union's bounds.
  std::vector<RectPiece> &pieces = ctx->fwd_pieces;
  pieces.clear();
  pieces.reserve(n);
  uint32_t acc = 0, x0 = W, y0 = H, x1 = 0, y1 = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const h266_rect &r = rects[i];
    if (r.x >= W || r.y >= H || !r.w || !r.h) continue;
    const uint32_t rw = (uint32_t)std::min<uint64_t>((uint64_t)r.x + r.w, W) - r.x;
    const uint32_t rh = (uint32_t)std::min<uint64_t>((uint64_t)r.y + r.h, H) - r.y;
    acc |= r.x | r.y | (r.x + rw) | (r.y + rh);
    x0 = std::min(x0, r.x);
    y0 = std::min(y0, r.y);
    x1 = std::max(x1, r.x + rw);
    y1 = std::max(y1, r.y + rh);
    pieces.push_back(RectPiece{r.x, r.y, rw, rh});
  }
  const uint32_t sh = grid_shift(acc);
  // Pieces of at most kPieceCells cells, split at rows of the grid.
  for (size_t i = 0, e = pieces.size(); i < e; ++i) {
    const RectPiece r = pieces[i];  // a copy: the appends below may move the array
    const uint32_t cols = r.w >> sh, rows = r.h >> sh;
    if ((uint64_t)cols * rows <= kPieceCells) continue;
    const uint32_t step = std::max<uint32_t>(1, kPieceCells / cols) << sh;
    for (uint32_t y = step; y < r.h; y += step)
      pieces.push_back(RectPiece{r.x, r.y + y, r.w, std::min(step, r.h - y)});
    pieces[i].h = step;
    if (pieces.size() > (1ull << 30)) return set_error(H266_ERR_UNSUPPORTED, "rectangles too large");
  }
  Guard g(ctx->device);
  Lane &ln = ctx->main;
  const h266_picture lv = plane_view(*pic, 0);
  DPlane P[3];
  H266_TRY(picture_to_device(ln, lv, P));
  ctx->h2d_bytes += host_plane_bytes(lv);
  const bool fresh = ln.fwd_ok && std::memcmp(&ln.fwd_key, lmcs, sizeof *lmcs) == 0;
  if (!fresh) {  // the table is rebuilt only when the LMCS parameters change
    ln.fwd_ok = false;
    H266_TRY(ln.fwd_lut.ensure(65536 * 2));
    H266_TRY(launch_lmcs_fwd_lut(ln.stream, ln.fwd_lut.as<uint16_t>(), *lmcs, &ctx->launches));
  }
  uint8_t *base = nullptr;
  H266_TRY(upload_raw(ln, pieces.data(), pieces.size() * sizeof(RectPiece), &base));
  ctx->h2d_bytes += pieces.size() * sizeof(RectPiece);
  FwdCover cov{};
  cov.sh = sh;
  cov.pitch = (W + (1u << sh) - 1) >> sh;
  const size_t cells = (size_t)cov.pitch * ((H + (1u << sh) - 1) >> sh);
  cov.x0 = x0;
  cov.y0 = y0;
  cov.x1 = x1;
  cov.y1 = y1;
  H266_TRY(ln.fwd_cover.ensure(16 + cells * 4, ln.stream));
  uint32_t *d_err = ln.fwd_cover.buf.as<uint32_t>();
  cov.cnt = d_err + 4;
  {
    Prof pf(ctx, ln.stream, H266_PROF_LMCS);
    H266_TRY(launch_lmcs_fwd_cover(ln.stream, P[0], ln.fwd_lut.as<uint16_t>(),
                                   reinterpret_cast<const RectPiece *>(base), (uint32_t)pieces.size(), cov,
                                   lmcs->bit_depth < 16, d_err, &ctx->launches));
  }
  H266_TRY(picture_from_device(ln, lv, false));
  ctx->d2h_bytes += host_plane_bytes(lv);
  uint32_t err = 0;
  H266_TRY(sync_read(ln, &err, d_err, 4));
  ln.fwd_key = *lmcs;
  ln.fwd_ok = true;
  if (!err) ln.fwd_cover.done();  // counters back at zero (a raised error word is cleared by the next call's fill)
  if (err) return set_error(H266_ERR_INVALID_ARGUMENT, "forward LMCS: a sample above (1 << BitDepth) - 1 has no bin");
  return H266_OK;
}

int h266_lmcs_chroma_var_scale(h266_ctx *ctx, const h266_picture *pic, const h266_lmcs_derived *lmcs, uint32_t mn,
                               uint32_t mx, uint32_t ctb_size_y, const h266_lmcs_cvs_block *blocks, uint64_t n,
                               uint32_t *var_scale) {
  H266_TRY(check_ctx(ctx));
  H266_TRY(check_picture(pic));
  if (!lmcs) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL lmcs");
  H266_TRY(check_lmcs(lmcs, mn, mx));
  if (n && (!blocks || !var_scale)) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL blocks / output");
  if (n > (1u << 26)) return set_error(H266_ERR_UNSUPPORTED, "too many blocks");
  const uint32_t size_y = std::min<uint32_t>(ctb_size_y, 64);
  if (!size_y || (size_y & (size_y - 1)))
    return set_error(H266_ERR_INVALID_ARGUMENT, "ctb_size_y must be a power of two");
  for (uint64_t i = 0; i < n; ++i) {  // the crate's reads stay inside the plane (src/ctu.rs:1789-1806)
    const h266_lmcs_cvs_block &b = blocks[i];
    if ((b.x_cu_cb > 0 && b.avail_l && b.x_cu_cb - 1 >= pic->luma.width) ||
        (b.y_cu_cb > 0 && b.avail_t && b.y_cu_cb - 1 >= pic->luma.height))
      return set_error(H266_ERR_INVALID_ARGUMENT, "CU origin outside the luma plane");
  }
  Guard g(ctx->device);
  Lane &ln = ctx->main;
  const h266_picture lv = plane_view(*pic, 0);
  DPlane P[3];
  H266_TRY(picture_to_device(ln, lv, P));
  ctx->h2d_bytes += host_plane_bytes(lv);
  Prep &pr = ctx_prep(ctx, 0);
  pr.blob.clear();
  Blob blob{pr.blob};
  const size_t off = blob.put(blocks, n * sizeof(h266_lmcs_cvs_block));
  uint8_t *base = nullptr;
  H266_TRY(upload_blob(ln, pr.blob, &base));
  ctx->h2d_bytes += pr.blob.size();
  H266_TRY(ln.walk.ensure(std::max<uint64_t>(n, 1) * 4));
  CvsTables t;
  for (int i = 0; i < 17; ++i) t.pivot[i] = lmcs->lmcs_pivot[i];
  for (int i = 0; i < 16; ++i) t.chroma_scale[i] = lmcs->chroma_scale_coeff[i];
  t.mn = mn;
  t.mx = mx;
  t.bd = lmcs->bit_depth;
  {
    Prof pf(ctx, ln.stream, H266_PROF_LMCS);
    H266_TRY(launch_lmcs_cvs(ln.stream, P[0], reinterpret_cast<const h266_lmcs_cvs_block *>(base + off), (uint32_t)n,
                             (int)size_y, t, ln.walk.as<uint32_t>(), &ctx->launches));
  }
  if (n) H266_TRY(sync_read(ln, var_scale, ln.walk.as<uint32_t>(), n * 4));
  ctx->d2h_bytes += n * 4;
  return H266_OK;
}

int h266_lmcs_add_chroma_residual(h266_ctx *ctx, h266_picture *pic, uint32_t bd, const int32_t *res, uint64_t n_res,
                                  const h266_chroma_res_block *blocks, uint64_t n) {
  H266_TRY(check_ctx(ctx));
  H266_TRY(check_picture(pic));
  if (bd < 8 || bd > 16) return set_error(H266_ERR_INVALID_ARGUMENT, "bit_depth must be 8..16");
  if (n && (!blocks || !res)) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL blocks / residuals");
  if (n >= 0xFFFFFFFFull) return set_error(H266_ERR_UNSUPPORTED, "too many residual blocks");
  const h266_plane *cp[2] = {&pic->cb, &pic->cr};
  uint32_t acc = 0, bx0[2] = {UINT32_MAX, UINT32_MAX}, by0[2] = {UINT32_MAX, UINT32_MAX}, bx1[2] = {0, 0},
           by1[2] = {0, 0};
  for (uint64_t i = 0; i < n; ++i) {
    const h266_chroma_res_block &b = blocks[i];
    if (b.plane != 1 && b.plane != 2) return set_error(H266_ERR_INVALID_ARGUMENT, "residual block plane must be 1 or 2");
    const h266_plane &pl = *cp[b.plane - 1];
    // src/ctu.rs:9931-9937 (the crate's planes have stride == width)
    if ((uint64_t)b.x + b.w > pl.width || (uint64_t)b.y + b.h > pl.height)
      return set_error(H266_ERR_INVALID_ARGUMENT, "chroma TB does not fit in the plane");
    if (b.res_offset > n_res || (uint64_t)b.w * b.h > n_res - b.res_offset)
      return set_error(H266_ERR_INVALID_ARGUMENT, "chroma TB residuals run past n_res");
    acc |= b.x | b.y | b.w | b.h;
    if (!b.w || !b.h) continue;
    const int k = b.plane - 1;
    bx0[k] = std::min(bx0[k], b.x);
    by0[k] = std::min(by0[k], b.y);
    bx1[k] = std::max(bx1[k], b.x + b.w);
    by1[k] = std::max(by1[k], b.y + b.h);
  }
  const uint32_t sh = grid_shift(acc);
  Guard g(ctx->device);
  Lane &ln = ctx->main;
  const h266_picture cv = plane_view(*pic, -1);
  DPlane P[3];
  H266_TRY(picture_to_device(ln, cv, P));
  ctx->h2d_bytes += host_plane_bytes(cv);
  const int32_t *d_res = res;
  if (pic->mem == H266_MEM_HOST && n_res) {
    H266_TRY(ln.scratch[0].ensure(n_res * 4));
    H266_CUDA(cudaMemcpyAsync(ln.scratch[0].ptr, res, n_res * 4, cudaMemcpyHostToDevice, ln.stream));
    d_res = ln.scratch[0].as<int32_t>();
    ctx->h2d_bytes += n_res * 4;
  }
  // Pairwise disjoint TBs (the usual list) take one owner pass and one add
  // pass in any order; the device reports an overlap, and then the add runs
  // as ordered launches of disjoint TBs instead.
  uint8_t *base = nullptr;
  H266_TRY(upload_raw(ln, blocks, n * sizeof(h266_chroma_res_block), &base));
  ctx->h2d_bytes += n * sizeof(h266_chroma_res_block);
  ResCover c{};
  c.sh = sh;
  size_t cells[2];
  for (int k = 0; k < 2; ++k) {
    const uint32_t gsz = 1u << sh;
    c.pitch[k] = (cp[k]->width + gsz - 1) >> sh;
    cells[k] = (size_t)c.pitch[k] * ((cp[k]->height + gsz - 1) >> sh);
    c.x0[k] = bx1[k] ? bx0[k] : 0;
    c.y0[k] = by1[k] ? by0[k] : 0;
    c.x1[k] = bx1[k];
    c.y1[k] = by1[k];
  }
  H266_TRY(ln.res_cover.ensure(16 + (cells[0] + cells[1]) * 4, ln.stream));
  uint32_t *d_overlap = ln.res_cover.buf.as<uint32_t>();
  c.own[0] = d_overlap + 4;
  c.own[1] = c.own[0] + cells[0];
  {
    Prof pf(ctx, ln.stream, H266_PROF_LMCS);
    H266_TRY(launch_chroma_residual_cover(ln.stream, P[1], P[2], reinterpret_cast<const h266_chroma_res_block *>(base),
                                          (uint32_t)n, d_res, (int)bd, c, d_overlap, &ctx->launches));
  }
  H266_TRY(picture_from_device(ln, cv, false));
  uint32_t overlap = 0;
  H266_TRY(sync_read(ln, &overlap, d_overlap, 4));
  ctx->d2h_bytes += host_plane_bytes(cv);
  if (!overlap) {
    ln.res_cover.done();  // owners cleared by the add pass
    return H266_OK;
  }
  // Ordered launches: the host splits the list into runs of pairwise
  // disjoint TBs with a coverage bitmap; the planes are as they came in.
  Coverage cov[2];
  cov[0].reset(pic->cb.width, pic->cb.height, sh);
  cov[1].reset(pic->cr.width, pic->cr.height, sh);
  std::vector<ResPiece> &pieces = ctx->res_pieces;
  pieces.clear();
  pieces.reserve(n);
  std::vector<uint32_t> group_end;
  for (uint64_t i = 0; i < n; ++i) {
    const h266_chroma_res_block &b = blocks[i];
    if (!b.w || !b.h) continue;
    Coverage &cc = cov[b.plane - 1];
    if (!cc.claim(b.x, b.y, b.w, b.h)) {  // overlaps a TB of the open launch: a new launch, in list order
      group_end.push_back((uint32_t)pieces.size());
      cov[0].clear();
      cov[1].clear();
      cc.claim(b.x, b.y, b.w, b.h);
    }
    const uint32_t rows = std::max<uint32_t>(1, kPieceSamples / b.w);
    for (uint32_t y = 0; y < b.h; y += rows)
      pieces.push_back(ResPiece{b.x, b.y + y, b.w, std::min(rows, b.h - y), b.plane, b.var_scale,
                                b.res_offset + (uint64_t)y * b.w, b.w, 0});
  }
  group_end.push_back((uint32_t)pieces.size());
  H266_TRY(upload_raw(ln, pieces.data(), pieces.size() * sizeof(ResPiece), &base));
  ctx->h2d_bytes += pieces.size() * sizeof(ResPiece);
  {
    Prof pf(ctx, ln.stream, H266_PROF_LMCS);
    uint32_t g0 = 0;
    for (uint32_t ge : group_end) {
      H266_TRY(launch_chroma_residual(ln.stream, P[1], P[2], reinterpret_cast<const ResPiece *>(base) + g0, ge - g0,
                                      d_res, (int)bd, &ctx->launches));
      g0 = ge;
    }
  }
  H266_TRY(picture_from_device(ln, cv));
  ctx->d2h_bytes += host_plane_bytes(cv);
  if (pic->mem == H266_MEM_DEVICE) H266_CUDA(cudaStreamSynchronize(ln.stream));
  return H266_OK;
}

int h266_output_convert(h266_ctx *ctx, const h266_picture *pic, const h266_crop_window *crop, uint32_t cfi,
                        uint32_t bd, void *dst, uint64_t cap, uint32_t dst_mem, uint64_t *written) {
  H266_TRY(check_ctx(ctx));
  H266_TRY(check_picture(pic));
  if (!crop) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL crop");
  if (dst_mem != H266_MEM_HOST && dst_mem != H266_MEM_DEVICE)
    return set_error(H266_ERR_INVALID_ARGUMENT, "dst_mem must be H266_MEM_HOST or H266_MEM_DEVICE");
  if (bd < 8 || bd > 16) return set_error(H266_ERR_INVALID_ARGUMENT, "bit_depth must be 8..16");
  const bool wide = bd > 8;
  OutPlanes o{};
  const uint32_t x0[3] = {crop->left, crop->left / 2, crop->left / 2}, y0[3] = {crop->top, crop->top / 2, crop->top / 2};
  const uint32_t w[3] = {crop->width, crop->width / 2, crop->width / 2};
  const uint32_t h[3] = {crop->height, crop->height / 2, crop->height / 2};
  const h266_plane *pl[3] = {&pic->luma, &pic->cb, &pic->cr};
  const int planes = cfi != 0 ? 3 : 1;
  for (int i = 0; i < planes; ++i) {  // the crate slices these rows (examples/decode_dump.rs:34)
    if ((uint64_t)x0[i] + w[i] > pl[i]->width || (uint64_t)y0[i] + h[i] > pl[i]->height)
      return set_error(H266_ERR_INVALID_ARGUMENT, "crop window outside the plane");
    o.x0[i] = x0[i];
    o.y0[i] = y0[i];
    o.w[i] = w[i];
    o.n[i] = (uint64_t)w[i] * h[i];
    o.total += o.n[i];
  }
  const uint64_t bytes = o.total * (wide ? 2 : 1);
  if (written) *written = bytes;
  if (!dst) return H266_OK;  // size query
  if (cap < bytes) return set_error(H266_ERR_INVALID_ARGUMENT, "dst smaller than the cropped dump");
  if (wide && dst_mem == H266_MEM_DEVICE && (reinterpret_cast<uintptr_t>(dst) & 1))
    return set_error(H266_ERR_INVALID_ARGUMENT, "device dst of a 16-bit dump must be 2-byte aligned");
  Guard g(ctx->device);
  Lane &ln = ctx->main;
  h266_picture v = *pic;
  if (planes == 1) v.cb.width = v.cb.height = v.cr.width = v.cr.height = 0;
  DPlane P[3];
  H266_TRY(picture_to_device(ln, v, P));
  ctx->h2d_bytes += host_plane_bytes(v);
  for (int i = 0; i < 3; ++i) o.p[i] = P[i];
  uint8_t *d_dst = static_cast<uint8_t *>(dst);
  if (dst_mem == H266_MEM_HOST) {
    H266_TRY(ln.walk.ensure(std::max<uint64_t>(bytes, 16)));
    d_dst = ln.walk.as<uint8_t>();
  }
  {
    Prof pf(ctx, ln.stream, H266_PROF_COPY);
    H266_TRY(launch_output_dump(ln.stream, o, d_dst, wide, &ctx->launches));
  }
  if (dst_mem == H266_MEM_HOST) {
    H266_TRY(sync_read(ln, dst, d_dst, bytes));
    ctx->d2h_bytes += bytes;
  }
  return H266_OK;
}

int h266_alf_decide_and_apply_clipped(h266_ctx *ctx, const h266_picture *src, h266_picture *rec,
                                      const h266_alf_aps_data *aps, uint32_t log2, uint32_t bd, uint32_t cfi,
                                      const uint32_t *col_bd, uint64_t n_col, const uint32_t *row_bd, uint64_t n_row,
                                      h266_alf_ctb *decisions, uint64_t n_decisions, uint64_t *sse) {
  H266_TRY(check_ctx(ctx));
  H266_TRY(check_picture(src));
  H266_TRY(check_picture(rec));
  if (!decisions) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL decisions");
  if (col_bd && !row_bd) return set_error(H266_ERR_INVALID_ARGUMENT, "row bounds NULL while col bounds are not");
  if (bd < 8 || bd > 14) return set_error(H266_ERR_UNSUPPORTED, "ALF trials need BitDepth 8..14");
  if (log2 < 5 || log2 > 7) return set_error(H266_ERR_UNSUPPORTED, "ALF trials need CtbLog2SizeY in 5..7");
  const uint32_t ctb = 1u << log2;
  const uint32_t wc = (rec->luma.width + ctb - 1) / ctb, hc = (rec->luma.height + ctb - 1) / ctb;
  const size_t n = (size_t)wc * hc;
  if (n_decisions != n) return set_error(H266_ERR_GRID_MISMATCH, "decisions size != CTB grid of rec");
  const bool aps_ok = aps && aps->alf_luma_filter_signal_flag;
  if (aps_ok && aps->n_luma_filters < 25)
    return set_error(H266_ERR_INVALID_ARGUMENT, "luma APS signals fewer than 25 filters");
  const int cols = aps ? 18 : 17, run = aps_ok ? 17 : 16;
  Guard g(ctx->device);
  Prep &pr = ctx_prep(ctx, 0);
  Pass2Host &h = pr.h;
  // The commit pass is apply_alf with luma only (the trial configuration,
  // src/alf_enc.rs:226-235); its CTB records get their sets from the decision.
  std::vector<h266_alf_ctb> all(n, h266_alf_ctb{});
  for (h266_alf_ctb &c : all) c.luma_on = 1;
  const h266_alf_picture ap{wc, hc, all.data()};
  const h266_alf_config cfg{1, 0, 0, 0, 0, bd, log2, cfi};
  h266_picture rl = *rec;  // luma only: chroma is neither read nor written
  rl.cb.width = rl.cb.height = rl.cr.width = rl.cr.height = 0;
  Pass2Inputs in;
  in.alf = &ap;
  in.alf_cfg = &cfg;
  in.cols = col_bd;
  in.rows = row_bd;
  in.n_cols = n_col;
  in.n_rows = n_row;
  H266_TRY(build_pass2(rl, in, h));
  // trial slots: fixed sets 0..15 (clipIdx 0), then the APS set
  h.luma_tab.assign((size_t)run * 600, 0);
  for (int t = 0; t < run; ++t)
    for (int c = 0; c < 25; ++c)
      for (int j = 0; j < 12; ++j) {
        int32_t *e = &h.luma_tab[(size_t)t * 600];
        e[c * 12 + j] = t < 16 ? kFixedSetCoeff[(t * 25 + c) * 12 + j] : aps->luma_coeff[c][j];
        e[300 + c * 12 + j] = alf_clip_value((int)bd, t < 16 ? 0 : aps->luma_clip_idx[c][j]);
      }
  if (!build_packed(h, (int)bd, 0, nullptr))
    return set_error(H266_ERR_UNSUPPORTED, "ALF trials: APS luma coefficients outside [-128, 127]");
  h.packed = true;
  Lane &ln = ctx->main;
  DPlane P[3], S[3];
  H266_TRY(picture_to_device(ln, rl, P));
  DPlane O;
  if (src->mem == H266_MEM_DEVICE) {
    O = dplane(src->luma, src->luma.samples, (int64_t)src->luma.stride);
  } else {
    const size_t row = (size_t)src->luma.width * 2;
    H266_TRY(ln.io[1].ensure(row * src->luma.height));
    H266_CUDA(cudaMemcpy2DAsync(ln.io[1].ptr, row, src->luma.samples, (size_t)src->luma.stride * 2, row,
                                src->luma.height, cudaMemcpyHostToDevice, ln.stream));
    O = dplane(src->luma, ln.io[1].as<uint16_t>(), src->luma.width);
    ctx->h2d_bytes += row * src->luma.height;
  }
  ctx->h2d_bytes += host_plane_bytes(rl);
  H266_TRY(ensure_scratch(ln, P, S));
  H266_TRY(plane_map(ctx, ln.stream, S[0], P[0], nullptr));  // the pre-ALF snapshot
  Staged st;
  pr.blob.clear();
  stage_pass2(h, pr.blob, st);
  H266_TRY(upload_blob(ln, pr.blob, &st.base));
  ctx->h2d_bytes += pr.blob.size();
  const size_t sse_bytes = n * cols * sizeof(unsigned long long);
  H266_TRY(ln.walk.ensure(sse_bytes + n * sizeof(int16_t)));
  auto *d_sse = ln.walk.as<unsigned long long>();
  auto *d_dec = reinterpret_cast<int16_t *>(ln.walk.as<uint8_t>() + sse_bytes);
  H266_CUDA(cudaMemsetAsync(d_sse, 0, sse_bytes, ln.stream));
  {
    Pass2Args a = h.args;
    bind_pass2(a, st.base, st, S, P);
    Prof pf(ctx, ln.stream, H266_PROF_SAO_ALF);
    H266_TRY(launch_alf_luma_trials(ln.stream, a, O, run, cols, d_sse, &ctx->launches));
    H266_TRY(launch_alf_luma_decide(ln.stream, reinterpret_cast<CtbDev *>(st.base + st.ctb), (int)n, d_sse, cols, run,
                                    d_dec, &ctx->launches));
  }
  H266_TRY(run_pass2(ctx, ln.stream, h.args, false, true, true, st.base, st, S, P));
  std::vector<int16_t> dec(n);
  H266_CUDA(cudaMemcpyAsync(dec.data(), d_dec, n * sizeof(int16_t), cudaMemcpyDeviceToHost, ln.stream));
  if (sse) H266_CUDA(cudaMemcpyAsync(sse, d_sse, sse_bytes, cudaMemcpyDeviceToHost, ln.stream));
  H266_TRY(picture_from_device(ln, rl));
  ctx->d2h_bytes += host_plane_bytes(rl) + n * sizeof(int16_t) + (sse ? sse_bytes : 0);
  for (size_t i = 0; i < n; ++i) {
    decisions[i] = h266_alf_ctb{};
    if (dec[i] < 0) continue;
    decisions[i].luma_on = 1;
    decisions[i].luma_filt_set_idx = (uint8_t)(dec[i] < 16 ? dec[i] : 16);
  }
  return H266_OK;
}

int h266_apply_in_loop_filters(h266_ctx *ctx, h266_picture *pic, const h266_in_loop_filter_args *args) {
  H266_TRY(check_ctx(ctx));
  H266_TRY(check_picture(pic));
  if (!args) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL args");
  Guard g(ctx->device);
  DPlane P[3];
  H266_TRY(picture_to_device(ctx->main, *pic, P));  // the copy overlaps the host-side preparation
  ctx->h2d_bytes += host_plane_bytes(*pic);
  H266_TRY(chain_on_device(ctx, *pic, P, *args));
  ctx->d2h_bytes += host_plane_bytes(*pic);
  return picture_from_device(ctx->main, *pic);
}

// Pictures of a batch are prepared on the worker pool (one picture per worker,
// in parallel) while this thread queues every prepared picture, in order, on
// one of kBatchLanes streams: upload, side information, chain, download.  The
// lanes start after the work already queued on the context stream, and the
// context stream waits for all of them before the call returns; host pictures
// are complete on return.

int h266_apply_in_loop_filters_batch(h266_ctx *ctx, uint32_t n, h266_picture *const *pics,
                                     const h266_in_loop_filter_args *const *args) {
  // Groups of pictures rotate over streams: per group the uploads (planes of
  // host pictures, side information staged in pinned memory by the worker
  // that prepared the picture), the LUTs, one batched execution (device
  // walks, tile deblocking, SAO / ALF) and the downloads.
  H266_TRY(check_ctx(ctx));
  if (n && (!pics || !args)) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL batch arrays");
  bool any_host = false;
  for (uint32_t i = 0; i < n; ++i) {
    H266_TRY(check_picture(pics[i]));
    if (!args[i]) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL args in batch");
    any_host |= pics[i]->mem == H266_MEM_HOST;
  }
  if (n <= 1) return n ? h266_apply_in_loop_filters(ctx, pics[0], args[0]) : H266_OK;
  Guard g(ctx->device);
  const Tuning &tn = batch_tuning(ctx, n, pics);
  const uint32_t kGroup = (uint32_t)tn.e2e_group, kGroupLanes = (uint32_t)tn.e2e_lanes;
  // Group boundaries.  With e2e_ramp the batch starts and ends with small
  // groups (1, 2, ... and ..., 2, 1 pictures): the first kernels and
  // downloads start after one picture's upload instead of a whole group's,
  // and the last group's kernels and downloads, which nothing overlaps, are
  // one picture's.
  std::vector<uint32_t> gb(1, 0);
  {
    std::vector<uint32_t> ramp;
    for (uint32_t g = 1; g < kGroup; g *= 2) ramp.push_back(g);
    uint32_t ends = 0;
    for (uint32_t g : ramp) ends += 2 * g;
    const bool use_ramp = tn.e2e_ramp && n >= ends + 2 * kGroup;
    uint32_t left = n;
    if (use_ramp)
      for (uint32_t g : ramp) {
        gb.push_back(gb.back() + g);
        left -= g;
      }
    const uint32_t tail = use_ramp ? ends / 2 : 0;
    while (left > tail) {
      const uint32_t g = std::min(kGroup, left - tail);
      gb.push_back(gb.back() + g);
      left -= g;
    }
    if (use_ramp)
      for (size_t k = ramp.size(); k-- > 0;) gb.push_back(gb.back() + ramp[k]);
  }
  const uint32_t n_groups = (uint32_t)gb.size() - 1, n_lanes = std::min(n_groups, kGroupLanes);
  for (auto &l : ctx->glanes)  // a larger group than the lanes were made for: more slots
    if (l->slots.size() < kGroup) l->slots.resize(kGroup);
  while (ctx->glanes.size() < n_lanes) {
    std::unique_ptr<GroupLane> l(new GroupLane());
    const int rc = l->init(kGroup);
    if (rc != H266_OK) {
      l->release();
      return rc;
    }
    ctx->glanes.push_back(std::move(l));
  }
  H266_CUDA(cudaEventRecord(ctx->main.mark, ctx->stream));
  for (uint32_t l = 0; l < n_lanes; ++l) H266_CUDA(cudaStreamWaitEvent(ctx->glanes[l]->stream, ctx->main.mark, 0));
  for (uint32_t i = 0; i < n; ++i) ctx_prep(ctx, i + 1);
  TaskPool *pool = ctx_pool(ctx);
  const int device = ctx->device;
  const bool allow_dev = device_sideinfo_allowed(ctx);
  using HClock = std::chrono::steady_clock;
  auto ns_since = [](HClock::time_point t0) {
    return (int64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(HClock::now() - t0).count();
  };
  pool->start(n, [&](size_t i) {
    const auto t0 = HClock::now();
    Prep &pr = *ctx->preps[i + 1];
    pr.staged_pinned = false;
    pr.rc = prepare_chain(pr, *pics[i], *args[i], nullptr, allow_dev);
    if (pr.rc == H266_OK && cudaSetDevice(device) == cudaSuccess) pr.rc = pr.stage();
    if (pr.rc != H266_OK) pr.msg = h266_last_error();
    ctx->host_ns[0] += ns_since(t0);
  });
  const bool copy_streams = tn.e2e_copy_streams != 0 && any_host;
  if (copy_streams) {
    for (cudaStream_t *st : {&ctx->e2e_up, &ctx->e2e_down}) {
      if (!*st) H266_CUDA(cudaStreamCreateWithFlags(st, cudaStreamNonBlocking));
      H266_CUDA(cudaStreamWaitEvent(*st, ctx->main.mark, 0));
    }
  }
  auto run_group = [&](uint32_t gi) -> int {
    GroupLane &L = *ctx->glanes[gi % n_lanes];
    std::vector<BatchItem> items;
    const uint32_t i0 = gb[gi], i1 = gb[gi + 1];
    // uploads on the upload stream once the lane's previous downloads freed its slots
    const cudaStream_t up = copy_streams ? ctx->e2e_up : L.stream;
    if (copy_streams) H266_CUDA(cudaStreamWaitEvent(up, L.ev_down, 0));
    // the planes first: they need no preparation, so the link starts at once
    items.resize(i1 - i0);
    for (uint32_t i = i0; i < i1; ++i) {
      GroupSlot &sl = L.slots[i - i0];
      const h266_picture &pic = *pics[i];
      BatchItem &it = items[i - i0];
      const h266_plane *pl[3] = {&pic.luma, &pic.cb, &pic.cr};
      for (int k = 0; k < 3; ++k) {
        const h266_plane &q = *pl[k];
        if (pic.mem == H266_MEM_DEVICE || (uint64_t)q.width * q.height == 0) {
          it.P[k] = dplane(q, q.samples, (int64_t)std::max<uint64_t>(q.stride, 1));
          continue;
        }
        const size_t row = (size_t)q.width * 2;
        H266_TRY(sl.io[k].ensure(row * q.height));
        if ((size_t)q.stride * 2 == row)  // contiguous rows: one linear copy
          H266_CUDA(cudaMemcpyAsync(sl.io[k].ptr, q.samples, row * q.height, cudaMemcpyHostToDevice, up));
        else
          H266_CUDA(cudaMemcpy2DAsync(sl.io[k].ptr, row, q.samples, (size_t)q.stride * 2, row, q.height,
                                      cudaMemcpyHostToDevice, up));
        it.P[k] = dplane(q, sl.io[k].as<uint16_t>(), q.width);
      }
      ctx->h2d_bytes += host_plane_bytes(pic);
    }
    // then each picture's side information once its worker has prepared it
    for (uint32_t i = i0; i < i1; ++i) {
      const auto tw = HClock::now();
      pool->wait_item(i);
      ctx->host_ns[1] += ns_since(tw);
      Prep &pr = *ctx->preps[i + 1];
      if (pr.rc != H266_OK) return set_error(pr.rc, pr.msg);
      GroupSlot &sl = L.slots[i - i0];
      const h266_in_loop_filter_args &a = *args[i];
      BatchItem &it = items[i - i0];
      H266_TRY(sl.side.ensure(pr.blob.size()));
      H266_CUDA(cudaMemcpyAsync(sl.side.ptr, pr.pinned.ptr, pr.blob.size(), cudaMemcpyHostToDevice, up));
      H266_CUDA(cudaEventRecord(pr.uploaded, up));
      ctx->h2d_bytes += pr.blob.size();
      it.st = pr.st;
      it.st.base = sl.side.as<uint8_t>();
      it.db = pr.db;
      it.args = pr.h.args;
      it.pass2 = pr.h.do_sao || pr.h.do_alf;
      it.do_sao = pr.h.do_sao;
      it.do_alf = pr.h.do_alf;
      it.packed = pr.h.packed;
      it.bd = (int)a.deblock.bit_depth;
      if (a.lmcs) {
        H266_TRY(sl.lut.ensure(65536 * 2));
        H266_TRY(build_lut(ctx, L.stream, sl.lut.as<uint16_t>(), *a.lmcs, a.lmcs_min_bin_idx, a.lmcs_max_bin_idx));
        it.lut = sl.lut.as<uint16_t>();
      }
      for (int k = 0; k < 3; ++k) {
        if (it.pass2) {
          const size_t np = (size_t)std::max(it.P[k].w, 0) * std::max(it.P[k].h, 0);
          H266_TRY(sl.scratch[k].ensure(std::max<size_t>(np, 1) * 2));
        }
        it.S[k] = DPlane{it.pass2 ? sl.scratch[k].as<uint16_t>() : nullptr, std::max(it.P[k].w, 1), it.P[k].w,
                         it.P[k].h};
      }
      if (pr.db.device_walk) {
        H266_TRY(sl.walk.ensure(device_walk_bytes(pr.db.dw)));
        it.walk = sl.walk.as<uint8_t>();
      }
    }
    if (copy_streams) {
      H266_CUDA(cudaEventRecord(L.ev_up, up));
      H266_CUDA(cudaStreamWaitEvent(L.stream, L.ev_up, 0));
    }
    H266_TRY(exec_batch(ctx, L.bb, L.stream, items, tn, copy_streams ? up : nullptr));
    const cudaStream_t down = copy_streams ? ctx->e2e_down : L.stream;
    if (copy_streams) {
      H266_CUDA(cudaEventRecord(L.ev_comp, L.stream));
      H266_CUDA(cudaStreamWaitEvent(down, L.ev_comp, 0));
    }
    for (uint32_t i = i0; i < i1; ++i) {
      const h266_picture &pic = *pics[i];
      if (pic.mem == H266_MEM_DEVICE) continue;
      GroupSlot &sl = L.slots[i - i0];
      const h266_plane *pl[3] = {&pic.luma, &pic.cb, &pic.cr};
      for (int k = 0; k < 3; ++k) {
        const h266_plane &q = *pl[k];
        if ((uint64_t)q.width * q.height == 0) continue;
        const size_t row = (size_t)q.width * 2;
        if ((size_t)q.stride * 2 == row)
          H266_CUDA(cudaMemcpyAsync(q.samples, sl.io[k].ptr, row * q.height, cudaMemcpyDeviceToHost, down));
        else
          H266_CUDA(cudaMemcpy2DAsync(q.samples, (size_t)q.stride * 2, sl.io[k].ptr, row, row, q.height,
                                      cudaMemcpyDeviceToHost, down));
      }
      ctx->d2h_bytes += host_plane_bytes(pic);
    }
    if (copy_streams) H266_CUDA(cudaEventRecord(L.ev_down, down));
    return H266_OK;
  };
  int rc = H266_OK;
  const auto ti = HClock::now();
  for (uint32_t gi = 0; gi < n_groups && rc == H266_OK; ++gi) rc = run_group(gi);
  pool->wait_all();
  ctx->host_ns[2] += ns_since(ti);
  for (uint32_t l = 0; l < n_lanes; ++l) {
    GroupLane &L = *ctx->glanes[l];
    H266_CUDA(cudaEventRecord(L.mark, L.stream));
    H266_CUDA(cudaStreamWaitEvent(ctx->stream, L.mark, 0));
    if (any_host || rc != H266_OK) H266_CUDA(cudaStreamSynchronize(L.stream));
  }
  if (copy_streams)
    for (cudaStream_t st : {ctx->e2e_up, ctx->e2e_down}) {
      H266_CUDA(cudaEventRecord(ctx->main.mark, st));
      H266_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->main.mark, 0));
      H266_CUDA(cudaStreamSynchronize(st));
    }
  return rc;
}

static const h266::TuningKey *tuning_key(const char *key) {
  if (!key) return nullptr;
  for (const h266::TuningKey &k : h266::kTuningKeys)
    if (std::strcmp(k.name, key) == 0) return &k;
  return nullptr;
}

int h266_ctx_set_tuning(h266_ctx *ctx, const char *key, int64_t value) {
  H266_TRY(check_ctx(ctx));
  const h266::TuningKey *k = tuning_key(key);
  if (!k) return set_error(H266_ERR_INVALID_ARGUMENT, std::string("unknown tuning key ") + (key ? key : "(null)"));
  if (value < k->lo || value > k->hi) return set_error(H266_ERR_INVALID_ARGUMENT, std::string(key) + ": value out of range");
  ctx->tuning.*(k->field) = (int)value;
  for (auto &kv : ctx->tuning_for) kv.second.*(k->field) = (int)value;
  return H266_OK;
}

int h266_ctx_set_tuning_for(h266_ctx *ctx, uint32_t width, uint32_t height, uint32_t bit_depth, const char *key,
                            int64_t value) {
  H266_TRY(check_ctx(ctx));
  const h266::TuningKey *k = tuning_key(key);
  if (!k) return set_error(H266_ERR_INVALID_ARGUMENT, std::string("unknown tuning key ") + (key ? key : "(null)"));
  if (value < k->lo || value > k->hi) return set_error(H266_ERR_INVALID_ARGUMENT, std::string(key) + ": value out of range");
  const uint64_t g = (uint64_t)width << 32 | (uint64_t)(height & 0xFFFFFF) << 8 | (bit_depth & 0xFF);
  auto it = ctx->tuning_for.find(g);
  if (it == ctx->tuning_for.end()) it = ctx->tuning_for.emplace(g, ctx->tuning).first;
  it->second.*(k->field) = (int)value;
  return H266_OK;
}

int h266_ctx_get_tuning(const h266_ctx *ctx, const char *key, int64_t *value) {
  if (!ctx || !value) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL argument");
  const h266::TuningKey *k = tuning_key(key);
  if (!k) return set_error(H266_ERR_INVALID_ARGUMENT, std::string("unknown tuning key ") + (key ? key : "(null)"));
  *value = ctx->tuning.*(k->field);
  return H266_OK;
}

int h266_ctx_host_profile(h266_ctx *ctx, double ms[3]) {
  H266_TRY(check_ctx(ctx));
  if (!ms) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL out");
  for (int k = 0; k < 3; ++k) ms[k] = (double)ctx->host_ns[k].exchange(0) / 1e6;
  ms[2] -= ms[1];  // issuing excludes the waits
  return H266_OK;
}

int h266_ctx_set_profiling(h266_ctx *ctx, int on) {
  H266_TRY(check_ctx(ctx));
  ctx->prof = on != 0;
  return H266_OK;
}

int h266_ctx_profile(h266_ctx *ctx, double ms[H266_PROF_FAMILIES], uint64_t launches[H266_PROF_FAMILIES]) {
  H266_TRY(check_ctx(ctx));
  Guard g(ctx->device);
  H266_CUDA(cudaStreamSynchronize(ctx->stream));
  for (auto &e : ctx->ev_pending) {
    float t = 0;
    H266_CUDA(cudaEventElapsedTime(&t, e.second.first, e.second.second));
    ctx->prof_ms[e.first] += t;
    ctx->prof_n[e.first] += 1;
    ctx->ev_pool.push_back(e.second.first);
    ctx->ev_pool.push_back(e.second.second);
  }
  ctx->ev_pending.clear();
  for (int i = 0; i < H266_PROF_FAMILIES; ++i) {
    if (ms) ms[i] = ctx->prof_ms[i];
    if (launches) launches[i] = ctx->prof_n[i];
    ctx->prof_ms[i] = 0;
    ctx->prof_n[i] = 0;
  }
  return H266_OK;
}

int h266_chain_plan_create(h266_ctx *ctx, const h266_picture *pic, const h266_in_loop_filter_args *args,
                           h266_chain_plan **out) {
  return h266_chain_plan_create_ex(ctx, pic, args, 0, out);
}

int h266_chain_plan_device_sideinfo(const h266_chain_plan *plan) { return plan && plan->db.device_walk ? 1 : 0; }

int h266_sideinfo_mode(const h266_picture *pic, const h266_in_loop_filter_args *args) {
  if (!pic || !args) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL picture or args");
  if (args->n_cus && !args->cus) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL CU list with nonzero length");
  if (args->n_chroma_cus && !args->chroma_cus)
    return set_error(H266_ERR_INVALID_ARGUMENT, "NULL chroma CU list with nonzero length");
  return h266::device_walk_mode(*pic, args->cus, args->n_cus, args->chroma_cus, args->n_chroma_cus, args->deblock,
                                args->chroma_format_idc);
}

int h266_chain_plan_create_ex(h266_ctx *ctx, const h266_picture *pic, const h266_in_loop_filter_args *args,
                              uint32_t flags, h266_chain_plan **out) {
  H266_TRY(check_ctx(ctx));
  if (flags & ~H266_PLAN_DEVICE_SIDEINFO) return set_error(H266_ERR_INVALID_ARGUMENT, "unknown plan flags");
  if (!out || !args) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  if (!pic) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL picture");
  h266_picture geom = *pic;
  geom.mem = H266_MEM_DEVICE;
  h266_plane *gp[3] = {&geom.luma, &geom.cb, &geom.cr};
  for (h266_plane *p : gp) {  // only the geometry is used; give check_picture a stand-in pointer
    p->samples = reinterpret_cast<uint16_t *>(uintptr_t(16));
    if (p->stride < p->width) p->stride = p->width;
  }
  H266_TRY(check_picture(&geom));
  Guard g(ctx->device);
  Prep &pr = ctx_prep(ctx, 0);
  H266_TRY(prepare_chain(pr, geom, *args, ctx_pool(ctx),
                         (flags & H266_PLAN_DEVICE_SIDEINFO) != 0 && device_sideinfo_allowed(ctx)));
  h266_chain_plan *pl = new h266_chain_plan();
  pl->device = ctx->device;
  pl->geom = geom;
  auto fail = [&](int rc) {
    h266_chain_plan_destroy(pl);
    return rc;
  };
  int rc = pl->side.ensure(pr.blob.size());
  if (rc != H266_OK) return fail(rc);
  cudaError_t e = cudaMemcpy(pl->side.ptr, pr.blob.data(), pr.blob.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(cuda_error(e, "plan upload"));
  pl->lmcs = args->lmcs != nullptr;
  if (pl->lmcs) {
    if ((rc = pl->lut.ensure(65536 * 2)) != H266_OK) return fail(rc);
    if ((rc = build_lut(ctx, ctx->stream, pl->lut.as<uint16_t>(), *args->lmcs, args->lmcs_min_bin_idx,
                        args->lmcs_max_bin_idx)) != H266_OK)
      return fail(rc);
  }
  pl->pass2 = pr.h.do_sao || pr.h.do_alf;
  if (pl->pass2) {
    const h266_plane *sp[3] = {&geom.luma, &geom.cb, &geom.cr};
    for (int i = 0; i < 3; ++i)
      if ((rc = pl->scratch[i].ensure(std::max<size_t>((size_t)sp[i]->width * sp[i]->height, 1) * 2)) != H266_OK)
        return fail(rc);
  }
  if (pr.db.device_walk && (rc = pl->walk.ensure(device_walk_bytes(pr.db.dw))) != H266_OK) return fail(rc);
  pl->deblock_bd = (int)args->deblock.bit_depth;
  pl->db = pr.db;
  pl->st = pr.st;
  pl->st.base = nullptr;
  pl->packed = pr.h.packed;
  pl->args = pr.h.args;
  pl->do_sao = pr.h.do_sao;
  pl->do_alf = pr.h.do_alf;
  e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return fail(cuda_error(e, "plan LUT"));
  *out = pl;
  return H266_OK;
}

}  // extern "C"

namespace h266 {
// One plan on one device picture, queued on `stream` with per-kernel launches
// (no batch parameter tables); the caller has checked the pair.
int exec_plan_single(h266_ctx *ctx, cudaStream_t stream, h266_chain_plan *plan, h266_picture *pic) {
  DPlane P[3], S[3];
  H266_TRY(picture_to_device(ctx->main, *pic, P));
  for (int i = 0; i < 3; ++i)
    S[i] = DPlane{plan->pass2 ? plan->scratch[i].as<uint16_t>() : nullptr, std::max(P[i].w, 1), P[i].w, P[i].h};
  Staged st = plan->st;
  st.base = plan->side.as<uint8_t>();
  Pass2Host h;
  h.args = plan->args;
  h.do_sao = plan->do_sao;
  h.do_alf = plan->do_alf;
  h.packed = plan->packed;
  return exec_chain(ctx, stream, st.base, st, plan->db, h, plan->lmcs ? plan->lut.as<uint16_t>() : nullptr,
                    plan->deblock_bd, P, S, plan->walk.as<uint8_t>());
}
}  // namespace h266

extern "C" {

int h266_chain_plan_execute(h266_ctx *ctx, h266_chain_plan *plan, h266_picture *pic) {
  H266_TRY(check_ctx(ctx));
  if (!plan) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL plan");
  H266_TRY(check_picture(pic));
  if (pic->mem != H266_MEM_DEVICE) return set_error(H266_ERR_INVALID_ARGUMENT, "plans execute on device pictures");
  if (!same_geometry(*pic, plan->geom)) return set_error(H266_ERR_INVALID_ARGUMENT, "picture geometry differs from the plan");
  if (plan->device != ctx->device) return set_error(H266_ERR_INVALID_ARGUMENT, "plan belongs to another device");
  Guard g(ctx->device);
  return exec_plan_single(ctx, ctx->stream, plan, pic);
}


}  // extern "C"

namespace h266 {
int check_plan_batch(h266_ctx *ctx, uint32_t n, h266_chain_plan *const *plans, h266_picture *const *pics) {
  if (n && (!plans || !pics)) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL batch arrays");
  for (uint32_t i = 0; i < n; ++i) {
    if (!plans[i]) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL plan in batch");
    H266_TRY(check_picture(pics[i]));
    if (pics[i]->mem != H266_MEM_DEVICE) return set_error(H266_ERR_INVALID_ARGUMENT, "plans execute on device pictures");
    if (!same_geometry(*pics[i], plans[i]->geom))
      return set_error(H266_ERR_INVALID_ARGUMENT, "picture geometry differs from its plan");
    if (plans[i]->device != ctx->device) return set_error(H266_ERR_INVALID_ARGUMENT, "plan belongs to another device");
  }
  return H266_OK;
}


// Queues a batch of chain executions on `stream` with its parameter tables in
// `bb`: the device walks of the pictures that derive their side information
// on the device (three launches for all of them), one tile-deblocking launch
// and one SAO/ALF launch per kernel variant over every picture's tiles, and
// per picture whatever the batched kernels do not take.
// `upload`: the stream that carries the parameter table's upload (the
// end-to-end pipeline's upload stream, so that the table is copied in issue
// order with the planes instead of competing with them); `stream` by default.
int exec_batch(h266_ctx *ctx, BatchBufs &bb, cudaStream_t stream, std::vector<BatchItem> &items,
               const Tuning &tn, cudaStream_t upload) {
  const uint32_t n = (uint32_t)items.size();
  if (!n) return H266_OK;
  H266_TRY(bb.init());
  struct Run {
    bool tile, packed;
    int variant;
  };
  std::vector<Run> runs(n);
  std::vector<uint8_t> tile_params, walk_items;
  std::vector<uint32_t> tile_first(1, 0), walk_first[3] = {{0}, {0}, {0}};  // clear, CU map, walk CTAs
  WalkBatchCounts walk_total;
  const size_t wis = walk_batch_item_size();
  std::vector<Pass2Args> p2[kPass2Variants];
  std::vector<uint32_t> p2_first[kPass2Variants];
  const size_t tps = deblock_tile_params_size();
  for (uint32_t i = 0; i < n; ++i) {
    BatchItem &it = items[i];
    Run &r = runs[i];
    const uint8_t *base = it.st.base;
    r.tile = it.pass2 && (it.db.device_walk ? it.db.dw_tiles : it.db.tiles_ok) && !ctx->force_global_deblock &&
             !ctx->force_strip_deblock;
    if (r.tile && it.db.device_walk) {  // the side information is derived on the device first, batched
      DeviceWalkOut g;
      WalkBatchCounts c;
      walk_items.resize(walk_items.size() + wis);
      fill_walk_batch_item(walk_items.data() + walk_items.size() - wis, device_walk_in(base, it.st, it.db), it.walk, g,
                           c);
      walk_first[0].push_back(walk_first[0].back() + c.clear_ctas);
      walk_first[1].push_back(walk_first[1].back() + c.grid_ctas);
      walk_first[2].push_back(walk_first[2].back() + c.walk_ctas);
      walk_total.offsets = std::max(walk_total.offsets, c.offsets);
      tile_params.resize(tile_params.size() + tps);
      const uint32_t tc =
          fill_deblock_tile_params_grid(tile_params.data() + tile_params.size() - tps, it.P, it.S, it.lut, it.bd, g);
      tile_first.push_back(tile_first.back() + tc);
    } else if (r.tile) {
      const StripSide v{reinterpret_cast<const EdgeSeg *>(base + it.st.seg[0]),
                        reinterpret_cast<const uint32_t *>(base + it.st.comp[0]),
                        reinterpret_cast<const uint32_t *>(base + it.st.band[0])};
      const StripSide h{reinterpret_cast<const EdgeSeg *>(base + it.st.seg[1]),
                        reinterpret_cast<const uint32_t *>(base + it.st.comp[1]),
                        reinterpret_cast<const uint32_t *>(base + it.st.band[1])};
      tile_params.resize(tile_params.size() + tps);
      const uint32_t c = fill_deblock_tile_params(tile_params.data() + tile_params.size() - tps, it.P, it.S, it.lut,
                                                  it.bd, v, h, reinterpret_cast<const uint32_t *>(base + it.st.tile_bounds),
                                                  it.db.tb_off, it.db.n_bands, it.db.tiles_x, it.db.tiles_y);
      tile_first.push_back(tile_first.back() + c);
    }
    r.packed = it.pass2 && it.packed && !ctx->force_scalar;
    r.variant = -1;
    if (r.packed) {
      Pass2Args a = it.args;
      a.tile_h = tn.sao_alf_tile_h;
      bind_pass2(a, base, it.st, it.S, it.P);
      uint32_t c = 0;
      r.variant = pass2_packed_variant(a, it.do_sao, it.do_alf, &c);
      if (p2_first[r.variant].empty()) p2_first[r.variant].push_back(0);
      p2[r.variant].push_back(a);
      p2_first[r.variant].push_back(p2_first[r.variant].back() + c);
    }
  }
  // one upload of every batched launch's parameter table
  std::vector<uint8_t> &b = bb.blob;
  b.clear();
  Blob blob{b};
  const size_t off_tp = blob.put(tile_params.data(), tile_params.size());
  const size_t off_tf = blob.put(tile_first.data(), tile_first.size() * sizeof(uint32_t));
  const size_t off_wi = blob.put(walk_items.data(), walk_items.size());
  size_t off_wf[3];
  for (int k = 0; k < 3; ++k) off_wf[k] = blob.put(walk_first[k].data(), walk_first[k].size() * sizeof(uint32_t));
  size_t off_p2[kPass2Variants] = {0}, off_p2f[kPass2Variants] = {0};
  const uint32_t zero_queue[kPass2Variants] = {0};  // the persistent launches' item counters, zero at launch
  const size_t off_q = blob.put(zero_queue, sizeof zero_queue);
  for (int v = 0; v < kPass2Variants; ++v)
    if (!p2[v].empty()) {
      off_p2[v] = blob.put(p2[v].data(), p2[v].size() * sizeof(Pass2Args));
      off_p2f[v] = blob.put(p2_first[v].data(), p2_first[v].size() * sizeof(uint32_t));
    }
  H266_TRY(bb.side.ensure(b.size()));
  const cudaStream_t ups = upload ? upload : stream;
  if (!bb.capturing) {
    H266_CUDA(cudaStreamWaitEvent(ups, bb.done, 0));  // earlier batches read bb.side (any stream)
    H266_CUDA(cudaEventSynchronize(bb.staged));      // the previous upload has read the staging buffer
  }
  H266_TRY(bb.stage.ensure(b.size()));
  std::memcpy(bb.stage.ptr, b.data(), b.size());
  H266_CUDA(cudaMemcpyAsync(bb.side.ptr, bb.stage.ptr, b.size(), cudaMemcpyHostToDevice, ups));
  H266_CUDA(cudaEventRecord(bb.staged, ups));
  if (ups != stream) H266_CUDA(cudaStreamWaitEvent(stream, bb.staged, 0));
  const uint8_t *dside = bb.side.as<uint8_t>();
  // deblocking: per picture where the tile kernel does not apply, then the batched walks and tiles
  for (uint32_t i = 0; i < n; ++i) {
    BatchItem &it = items[i];
    if (runs[i].tile) continue;
    if (it.pass2) H266_TRY(run_deblock(ctx, stream, it.st.base, it.st, it.db, it.P, it.S, it.lut, it.bd, it.walk));
    else H266_TRY(run_deblock(ctx, stream, it.st.base, it.st, it.db, it.P, it.P, it.lut, it.bd, it.walk));
  }
  if (walk_first[0].size() > 1) {
    walk_total.clear_ctas = walk_first[0].back();
    walk_total.grid_ctas = walk_first[1].back();
    walk_total.walk_ctas = walk_first[2].back();
    Prof pf(ctx, stream, H266_PROF_DEBLOCK);
    H266_TRY(launch_walk_batch(stream, dside + off_wi, reinterpret_cast<const uint32_t *>(dside + off_wf[0]),
                               reinterpret_cast<const uint32_t *>(dside + off_wf[1]),
                               reinterpret_cast<const uint32_t *>(dside + off_wf[2]), (int)walk_first[0].size() - 1,
                               walk_total, &ctx->launches));
  }
  if (tile_first.size() > 1) {
    Prof pf(ctx, stream, H266_PROF_DEBLOCK);
    H266_TRY(launch_deblock_tiles_batch(stream, dside + off_tp, reinterpret_cast<const uint32_t *>(dside + off_tf),
                                        (int)tile_first.size() - 1, tile_first.back(), &ctx->launches));
  }
  // SAO / ALF: per picture where the packed kernel does not apply, then one launch per variant
  for (uint32_t i = 0; i < n; ++i) {
    BatchItem &it = items[i];
    if (!it.pass2 || runs[i].packed) continue;
    H266_TRY(run_pass2(ctx, stream, it.args, it.do_sao, it.do_alf, it.packed, it.st.base, it.st, it.S, it.P));
  }
  for (int v = 0; v < kPass2Variants; ++v)
    if (!p2[v].empty()) {
      Prof pf(ctx, stream, H266_PROF_SAO_ALF);
      H266_TRY(launch_pass2_packed_batch(stream, v, reinterpret_cast<const Pass2Args *>(dside + off_p2[v]),
                                         reinterpret_cast<const uint32_t *>(dside + off_p2f[v]), (int)p2[v].size(),
                                         p2_first[v].back(), tn.sao_alf_ctas_per_sm,
                                         reinterpret_cast<uint32_t *>(bb.side.as<uint8_t>() + off_q) + v,
                                         &ctx->launches));
    }
  H266_CUDA(cudaEventRecord(bb.done, stream));
  return H266_OK;
}

// Queues a batch of plan executions on `stream` with its parameter tables in
// `bb`; the caller has checked the batch and made the device current.
int exec_plan_batch(h266_ctx *ctx, BatchBufs &bb, cudaStream_t stream, uint32_t n, h266_chain_plan *const *plans,
                    h266_picture *const *pics) {
  if (!n) return H266_OK;
  std::vector<BatchItem> items(n);
  for (uint32_t i = 0; i < n; ++i) {
    const h266_chain_plan &pl = *plans[i];
    BatchItem &it = items[i];
    H266_TRY(picture_to_device(ctx->main, *pics[i], it.P));
    for (int k = 0; k < 3; ++k)
      it.S[k] = DPlane{pl.pass2 ? pl.scratch[k].as<uint16_t>() : nullptr, std::max(it.P[k].w, 1), it.P[k].w, it.P[k].h};
    it.st = pl.st;
    it.st.base = pl.side.as<uint8_t>();
    it.db = pl.db;
    it.args = pl.args;
    it.pass2 = pl.pass2;
    it.do_sao = pl.do_sao;
    it.do_alf = pl.do_alf;
    it.packed = pl.packed;
    it.lut = pl.lmcs ? pl.lut.as<uint16_t>() : nullptr;
    it.bd = pl.deblock_bd;
    it.walk = pl.walk.as<uint8_t>();
  }
  return exec_batch(ctx, bb, stream, items, batch_tuning(ctx, n, pics));
}
}  // namespace h266

extern "C" {

int h266_chain_plan_execute_batch(h266_ctx *ctx, uint32_t n, h266_chain_plan *const *plans,
                                  h266_picture *const *pics) {
  H266_TRY(check_ctx(ctx));
  H266_TRY(check_plan_batch(ctx, n, plans, pics));
  if (!n) return H266_OK;
  Guard g(ctx->device);
  return exec_plan_batch(ctx, ctx->batch, ctx->stream, n, plans, pics);
}

}  // extern "C"

// A batched plan execution recorded once as a CUDA graph: its own parameter
// tables (pinned staging and device copy, read by the graph's upload node on
// every replay) and the instantiated graph.
struct h266_batch_graph {
  int device = 0;
  h266::BatchBufs bb;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t stream = nullptr;  // the capture stream
};

extern "C" {

int h266_batch_graph_destroy(h266_batch_graph *g) {
  if (!g) return H266_OK;
  Guard gd(g->device);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->stream) cudaStreamDestroy(g->stream);
  g->bb.release();
  delete g;
  return H266_OK;
}

int h266_batch_graph_create(h266_ctx *ctx, uint32_t n, h266_chain_plan *const *plans, h266_picture *const *pics,
                            h266_batch_graph **out) {
  H266_TRY(check_ctx(ctx));
  if (!out) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL out");
  *out = nullptr;
  H266_TRY(check_plan_batch(ctx, n, plans, pics));
  if (!n) return set_error(H266_ERR_INVALID_ARGUMENT, "empty batch");
  Guard gd(ctx->device);
  h266_batch_graph *g = new h266_batch_graph();
  g->device = ctx->device;
  auto fail = [&](int rc) {
    h266_batch_graph_destroy(g);
    return rc;
  };
  int rc = g->bb.init();
  if (rc != H266_OK) return fail(rc);
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(cuda_error(e, "graph stream"));
  g->bb.capturing = true;
  const bool prof = ctx->prof;
  ctx->prof = false;  // no profiling events inside the graph
  // relaxed: the graph's own tables are allocated while recording
  e = cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) {
    ctx->prof = prof;
    return fail(cuda_error(e, "cudaStreamBeginCapture"));
  }
  rc = exec_plan_batch(ctx, g->bb, g->stream, n, plans, pics);
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(g->stream, &graph);
  ctx->prof = prof;
  g->graph = graph;
  if (rc != H266_OK) return fail(rc);
  if (e != cudaSuccess) return fail(cuda_error(e, "cudaStreamEndCapture"));
  e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (e != cudaSuccess) return fail(cuda_error(e, "cudaGraphInstantiate"));
  *out = g;
  return H266_OK;
}

int h266_batch_graph_launch(h266_ctx *ctx, h266_batch_graph *g) {
  H266_TRY(check_ctx(ctx));
  if (!g) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL graph");
  if (g->device != ctx->device) return set_error(H266_ERR_INVALID_ARGUMENT, "graph belongs to another device");
  Guard gd(ctx->device);
  H266_CUDA(cudaGraphLaunch(g->exec, ctx->stream));
  ctx->launches += 1;
  return H266_OK;
}

int h266_chain_plan_destroy(h266_chain_plan *plan) {
  if (!plan) return H266_OK;
  Guard g(plan->device);
  plan->side.release();
  plan->lut.release();
  plan->walk.release();
  for (auto &b : plan->scratch) b.release();
  delete plan;
  return H266_OK;
}

}  // extern "C"

// ======================================================================= served filter chain
//
// A request loop for many concurrent streams: callers submit (plan, device
// picture) requests from any thread; a dispatcher thread admits the queued
// requests into a batch as soon as one of kServerSlots batch slots is free and
// the device-memory budget allows, and queues the batch (one batched
// execution, h266_chain_plan_execute_batch's path) on that slot's stream.
// Batches of different slots overlap on the GPU, so requests that arrive while
// others are running start without waiting for them (continuous batching).
// A completion thread waits for the batches in order and records each
// request's latency from submission to completion.  max_batch = 1 gives plain
// per-picture launches of the same kernels.
namespace {

constexpr int kServerSlots = 3;
using Clock = std::chrono::steady_clock;

struct ServerReq {
  uint64_t ticket;
  h266_chain_plan *plan;
  h266_picture pic;
  uint64_t bytes;
  Clock::time_point t0;
};

struct ServerSlot {
  h266::BatchBufs bb;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  bool busy = false;
};

struct ServerFlight {
  std::vector<ServerReq> reqs;
  int slot;
  uint64_t bytes;
  int rc;
  std::string msg;
};

struct ServerResult {
  int rc;
  double ms;
  std::string msg;
};

}  // namespace

struct h266_server {
  h266_ctx *ctx = nullptr;  // the server's own context, used by the dispatcher thread only
  uint32_t max_batch = 1;
  // a batch grows past one request only while its luma samples stay within
  // this (0: no cap): a large picture is not held back by the small ones it
  // would share a batch with
  uint64_t batch_px = 1920ull * 1080;
  uint64_t budget = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_flight, cv_done;
  std::deque<ServerReq> queue;
  std::deque<ServerFlight> flights;
  ServerSlot slots[kServerSlots];
  std::unordered_map<uint64_t, ServerResult> results;
  std::unordered_set<uint64_t> pending;
  uint64_t next_ticket = 1, inflight = 0, batches = 0, requests = 0;
  bool stop = false, dispatcher_done = false;
  std::thread dispatcher, completer;
};

namespace {

int free_slot(const h266_server *s) {
  for (int i = 0; i < kServerSlots; ++i)
    if (!s->slots[i].busy) return i;
  return -1;
}

void server_dispatch(h266_server *s) {
  cudaSetDevice(s->ctx->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    s->cv_work.wait(lk, [&] { return (s->stop && s->queue.empty()) || (!s->queue.empty() && free_slot(s) >= 0); });
    if (s->queue.empty()) break;  // stopping and drained
    const int slot = free_slot(s);
    // admit in arrival order up to max_batch and the memory budget (an idle
    // server always admits the first request)
    std::vector<ServerReq> take;
    uint64_t bytes = 0, px = 0;
    while (!s->queue.empty() && take.size() < s->max_batch) {
      const ServerReq &r = s->queue.front();
      if ((s->inflight > 0 || !take.empty()) && s->inflight + bytes + r.bytes > s->budget) break;
      const uint64_t rpx = (uint64_t)r.pic.luma.width * r.pic.luma.height;
      if (!take.empty() && s->batch_px && px + rpx > s->batch_px) break;
      px += rpx;
      bytes += r.bytes;
      take.push_back(r);
      s->queue.pop_front();
    }
    if (take.empty()) {  // over budget: wait for a completion
      s->cv_work.wait(lk);
      continue;
    }
    s->slots[slot].busy = true;
    s->inflight += bytes;
    lk.unlock();
    std::vector<h266_chain_plan *> plans(take.size());
    std::vector<h266_picture *> pics(take.size());
    for (size_t i = 0; i < take.size(); ++i) {
      plans[i] = take[i].plan;
      pics[i] = &take[i].pic;
    }
    ServerSlot &sl = s->slots[slot];
    // one request: per-kernel launches, no batch tables to build and upload
    int rc = take.size() == 1 ? exec_plan_single(s->ctx, sl.stream, plans[0], pics[0])
                              : exec_plan_batch(s->ctx, sl.bb, sl.stream, (uint32_t)take.size(), plans.data(), pics.data());
    std::string msg = rc == H266_OK ? std::string() : std::string(h266_last_error());
    if (cudaEventRecord(sl.done, sl.stream) != cudaSuccess && rc == H266_OK) {
      rc = H266_ERR_CUDA;
      msg = "cudaEventRecord";
    }
    lk.lock();
    s->flights.push_back(ServerFlight{std::move(take), slot, bytes, rc, msg});
    ++s->batches;
    s->cv_flight.notify_one();
  }
  s->dispatcher_done = true;
  s->cv_flight.notify_all();
}

void server_complete(h266_server *s) {
  cudaSetDevice(s->ctx->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    s->cv_flight.wait(lk, [&] { return !s->flights.empty() || s->dispatcher_done; });
    if (s->flights.empty()) break;
    ServerFlight f = std::move(s->flights.front());
    s->flights.pop_front();
    lk.unlock();
    const cudaError_t e = cudaEventSynchronize(s->slots[f.slot].done);
    const Clock::time_point t1 = Clock::now();
    lk.lock();
    for (const ServerReq &r : f.reqs) {
      ServerResult res{f.rc, std::chrono::duration<double, std::milli>(t1 - r.t0).count(), f.msg};
      if (res.rc == H266_OK && e != cudaSuccess) {
        res.rc = H266_ERR_CUDA;
        res.msg = std::string("batch: ") + cudaGetErrorString(e);
      }
      s->results[r.ticket] = res;
      s->pending.erase(r.ticket);
    }
    s->requests += f.reqs.size();
    s->slots[f.slot].busy = false;
    s->inflight -= f.bytes;
    s->cv_done.notify_all();
    s->cv_work.notify_one();
  }
}

uint64_t request_bytes(const h266_picture &p, const h266_chain_plan &pl) {
  const h266_plane *q[3] = {&p.luma, &p.cb, &p.cr};
  uint64_t b = 0;
  for (const h266_plane *x : q) b += (uint64_t)x->width * x->height * 2;
  return pl.pass2 ? 2 * b : b;  // the picture's planes, plus the plan's scratch planes
}

}  // namespace

extern "C" {

int h266_server_create(int device, uint32_t max_batch, uint64_t memory_budget, h266_server **out) {
  if (!out) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL out");
  *out = nullptr;
  if (max_batch == 0) return set_error(H266_ERR_INVALID_ARGUMENT, "max_batch must be at least 1");
  h266_ctx *ctx = nullptr;
  H266_TRY(h266_ctx_create(device, &ctx));
  h266_server *s = new h266_server();
  s->ctx = ctx;
  s->max_batch = max_batch;
  s->budget = memory_budget;
  Guard g(device);
  // Parameter tables sized for a full batch up front: growing them later
  // would synchronise the device (and allocate pinned memory) mid-run.
  const size_t reserve = std::max<size_t>((size_t)max_batch * (deblock_tile_params_size() + sizeof(Pass2Args) + 64),
                                          256 * 1024);
  for (ServerSlot &sl : s->slots) {
    cudaError_t e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
    int rc = e == cudaSuccess ? sl.bb.init() : H266_OK;
    if (e == cudaSuccess && rc == H266_OK) rc = sl.bb.side.ensure(reserve);
    if (e == cudaSuccess && rc == H266_OK) rc = sl.bb.stage.ensure(reserve);
    if (e != cudaSuccess || rc != H266_OK) {
      h266_server_destroy(s);
      return e != cudaSuccess ? cuda_error(e, "h266_server_create") : rc;
    }
    sl.bb.blob.reserve(reserve);
  }
  s->dispatcher = std::thread(server_dispatch, s);
  s->completer = std::thread(server_complete, s);
  *out = s;
  return H266_OK;
}

int h266_server_submit(h266_server *s, h266_chain_plan *plan, h266_picture *pic, uint64_t *ticket) {
  if (!s || !ticket) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL server or ticket");
  H266_TRY(check_plan_batch(s->ctx, 1, &plan, &pic));
  ServerReq r{0, plan, *pic, request_bytes(*pic, *plan), Clock::now()};
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return set_error(H266_ERR_INVALID_ARGUMENT, "server is stopping");
  r.ticket = s->next_ticket++;
  s->pending.insert(r.ticket);
  s->queue.push_back(r);
  *ticket = r.ticket;
  s->cv_work.notify_one();
  return H266_OK;
}

int h266_server_wait(h266_server *s, uint64_t ticket, double *latency_ms) {
  if (!s) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL server");
  std::unique_lock<std::mutex> lk(s->mu);
  s->cv_done.wait(lk, [&] { return s->results.count(ticket) || !s->pending.count(ticket); });
  auto it = s->results.find(ticket);
  if (it == s->results.end()) return set_error(H266_ERR_INVALID_ARGUMENT, "unknown or already collected ticket");
  const ServerResult r = it->second;
  s->results.erase(it);
  if (latency_ms) *latency_ms = r.ms;
  if (r.rc != H266_OK) return set_error(r.rc, r.msg);
  return H266_OK;
}

int h266_server_stats(h266_server *s, uint64_t *requests, uint64_t *batches) {
  if (!s) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  if (requests) *requests = s->requests;
  if (batches) *batches = s->batches;
  return H266_OK;
}

int h266_server_replay(h266_server *s, uint32_t n, h266_chain_plan *const *plans, h266_picture *const *pics,
                       const double *arrival_s, const int32_t *after, double *latency_ms) {
  if (!s || (n && (!plans || !pics || !arrival_s || !latency_ms)))
    return set_error(H266_ERR_INVALID_ARGUMENT, "NULL argument");
  for (uint32_t i = 0; i < n; ++i) {
    if (i && arrival_s[i] < arrival_s[i - 1]) return set_error(H266_ERR_INVALID_ARGUMENT, "arrivals not in order");
    if (after && after[i] >= (int32_t)i) return set_error(H266_ERR_INVALID_ARGUMENT, "after[i] must precede i");
  }
  std::vector<uint64_t> tickets(n, 0);
  std::vector<std::atomic<int>> state(n);  // 0 not submitted, 1 submitted, 2 done
  for (auto &x : state) x.store(0);
  std::vector<Clock::time_point> due(n);
  std::atomic<uint32_t> submitted{0};
  std::atomic<int> first_rc{H266_OK};
  std::string first_msg;
  std::mutex msg_mu;
  // completions in submission order on a second thread
  std::thread collector([&] {
    for (uint32_t i = 0; i < n; ++i) {
      while (submitted.load(std::memory_order_acquire) <= i) {
        if (first_rc.load() != H266_OK && submitted.load() <= i) return;
        std::this_thread::yield();
      }
      double ms = 0;
      const int rc = h266_server_wait(s, tickets[i], &ms);
      latency_ms[i] = std::chrono::duration<double, std::milli>(Clock::now() - due[i]).count();
      if (rc != H266_OK && first_rc.load() == H266_OK) {
        std::lock_guard<std::mutex> lk(msg_mu);
        first_msg = h266_last_error();
        first_rc.store(rc);
      }
      state[i].store(2, std::memory_order_release);
    }
  });
  const Clock::time_point t0 = Clock::now();
  int rc = H266_OK;
  for (uint32_t i = 0; i < n; ++i) {
    due[i] = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[i]));
    while (Clock::now() < due[i]) {
    }
    if (after && after[i] >= 0)
      while (state[after[i]].load(std::memory_order_acquire) != 2) std::this_thread::yield();
    rc = h266_server_submit(s, plans[i], pics[i], &tickets[i]);
    if (rc != H266_OK) {
      std::lock_guard<std::mutex> lk(msg_mu);
      if (first_rc.load() == H266_OK) {
        first_msg = h266_last_error();
        first_rc.store(rc);
      }
      break;
    }
    state[i].store(1);
    submitted.store(i + 1, std::memory_order_release);
  }
  collector.join();
  if (first_rc.load() != H266_OK) return set_error(first_rc.load(), first_msg);
  return H266_OK;
}

int h266_server_set_batch_pixels(h266_server *s, uint64_t px) {
  if (!s) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->batch_px = px;
  return H266_OK;
}

int h266_server_destroy(h266_server *s) {
  if (!s) return H266_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->dispatcher.joinable()) s->dispatcher.join();
  if (s->completer.joinable()) s->completer.join();
  if (s->ctx) {
    Guard g(s->ctx->device);
    for (ServerSlot &sl : s->slots) {
      if (sl.stream) cudaStreamSynchronize(sl.stream);
      sl.bb.release();
      if (sl.done) cudaEventDestroy(sl.done);
      if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    h266_ctx_destroy(s->ctx);
  }
  delete s;
  return H266_OK;
}

}  // extern "C"

// ======================================================================= allocation-free chain
//
// For callers that must not allocate device memory at run time: real-time
// decode loops that forbid allocator calls (and their latency) once streaming
// has started, and hosts that hand the whole device budget to their own pool,
// where a library allocation would fail or escape their accounting.  The
// chain's scratch --
// the side information of the call, the LMCS LUT and the deblocked planes the
// SAO / ALF pass reads -- lives in this fixed device array instead of in a
// context.  Every GPU that loads the library holds the array until the process
// exits.
namespace {

static __device__ __align__(256) uint8_t g_noalloc_scratch[H266_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch on the current device.  In host code the
// symbol is only a host-side stand-in, so the address is looked up with the
// device current -- on every call, not cached: a cached address would outlive
// a cudaDeviceReset or a recreated primary context.  The lookup allocates
// nothing; the first one on a device also loads this library's device code.
int noalloc_scratch(uint8_t **out) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
  *out = static_cast<uint8_t *>(p);
  return H266_OK;
}

inline size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

}  // namespace

extern "C" int h266_apply_in_loop_filters_noalloc(h266_picture *pic, const h266_in_loop_filter_args *args,
                                                  void *cuda_stream) {
  H266_TRY(check_picture(pic));
  if (!args) return set_error(H266_ERR_INVALID_ARGUMENT, "NULL args");
  if (pic->mem != H266_MEM_DEVICE)
    return set_error(H266_ERR_INVALID_ARGUMENT, "the allocation-free chain takes device planes (H266_MEM_DEVICE)");
  uint8_t *scratch = nullptr;
  H266_TRY(noalloc_scratch(&scratch));
  // A context object on the stack carries the stream and the launch counter;
  // it owns no device memory and no CUDA handles.  The side information is
  // built on this thread.
  h266_ctx local;
  H266_CUDA(cudaGetDevice(&local.device));
  local.stream = (cudaStream_t)cuda_stream;
  Prep pr;
  H266_TRY(prepare_chain(pr, *pic, *args, nullptr));
  // Scratch layout: [side information][LMCS LUT][three deblocked planes].
  const size_t blob = align256(pr.blob.size());
  const size_t lut_off = blob, lut_bytes = args->lmcs ? align256(65536 * 2) : 0;
  size_t planes_off = lut_off + lut_bytes, need = planes_off;
  const bool pass2 = pr.h.do_sao || pr.h.do_alf;
  const h266_plane *pl[3] = {&pic->luma, &pic->cb, &pic->cr};
  size_t plane_off[3] = {0, 0, 0};
  for (int i = 0; i < 3; ++i) {
    plane_off[i] = need;
    if (pass2) need += align256((size_t)pl[i]->width * pl[i]->height * 2);
  }
  if (need > H266_NOALLOC_SCRATCH_BYTES)
    return set_error(H266_ERR_UNSUPPORTED, "picture needs " + std::to_string(need) +
                                               " bytes of scratch; the allocation-free chain has " +
                                               std::to_string((size_t)H266_NOALLOC_SCRATCH_BYTES));
  // Every scratch region is written in full below before anything reads it,
  // so no region needs clearing.
  if (!pr.blob.empty())
    H266_CUDA(cudaMemcpyAsync(scratch, pr.blob.data(), pr.blob.size(), cudaMemcpyHostToDevice, local.stream));
  pr.st.base = scratch;
  const uint16_t *lut = nullptr;
  if (args->lmcs) {
    uint16_t *l = reinterpret_cast<uint16_t *>(scratch + lut_off);
    H266_TRY(build_lut(&local, local.stream, l, *args->lmcs, args->lmcs_min_bin_idx, args->lmcs_max_bin_idx));
    lut = l;
  }
  DPlane P[3], S[3];
  for (int i = 0; i < 3; ++i) {
    P[i] = dplane(*pl[i], pl[i]->samples, (int64_t)std::max<uint64_t>(pl[i]->stride, 1));
    S[i] = DPlane{reinterpret_cast<uint16_t *>(scratch + plane_off[i]), std::max<int>((int)pl[i]->width, 1),
                  (int)pl[i]->width, (int)pl[i]->height};
  }
  return exec_chain(&local, local.stream, scratch, pr.st, pr.db, pr.h, lut, (int)args->deblock.bit_depth, P, S);
}
