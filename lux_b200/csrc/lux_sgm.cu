// C ABI of the dense-stereo depth stage (include/lux_sgm.h): contexts, device memory under an HBM budget, one layer,
// the six-layer pyramid, and the upsample. The seams are DenseStereoPyramid.Run / DenseLayer (DenseStereoSgm.cs:331,
// 34, 181) and DenseUpsampleLayer.Run (DenseUpsampleLayer.cs:35).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/lux_sgm.h"
#include "host_geom.h"
#include "internal.h"
#include "revisit_schedule.h"

using namespace lux;

struct lux_sgm_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint64_t budget = 0;
  uint64_t in_use = 0;
  std::mutex mu;
  std::string last_error;
  uint32_t* d_rcp = nullptr;  // 4096-entry rcp table
  uint32_t* d_skip_bits = nullptr;  // the skip mask's generator stream (host_skip_stream_bits)
  uint32_t* d_warp = nullptr; // the rsqrt tables (exponents 127, 128; 4096 entries each), then the 384-float Lanczos table
  int* d_err = nullptr;       // device error word of the current call
  cudaEvent_t ev[4] = {};
  uint64_t wait_limit_ns = kTimeoutNs;  // bound of every device-side wait of the aggregation kernels
  int stall_block = -1;                 // failure-path tests: the block whose cross-block wait can never be satisfied
  int* d_never = nullptr;               // the zero counter that block waits on (nothing writes it)
  bool autotune = true;                 // untuned layer shapes time every fast form on their first solve
};

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// The autotuner's choices, per layer shape (W, H, planes, tile), shared by every context of the process: the fast
// aggregation form (1 fused wavefront, 2 path-group chains, 3 lean wavefront) measured fastest on the first solve of
// that shape.
namespace {
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, int> g_tuned;
int tuned_form(int W, int H, int n, int T) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tuned.find(std::make_tuple(W, H, n, T));
  return it == g_tuned.end() ? 0 : it->second;
}
void set_tuned_form(int W, int H, int n, int T, int form) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (form) g_tuned[std::make_tuple(W, H, n, T)] = form;
  else g_tuned.erase(std::make_tuple(W, H, n, T));
}
}  // namespace

struct lux_layer {
  lux_sgm_ctx* ctx = nullptr;
  int w = 0, h = 0, index = 0, align = 8, n = 0, min_lo = 0, max_hi = 0, tile = 4;
  uint64_t volume = 0;
  float ms_cost = 0.f, ms_sgm = 0.f, ms_wta = 0.f;
  int sgm_kernel = 0;
  int cost_kernel = 0;
  int tuned = 0;  // the form the autotuner chose on this solve (0: no tuning ran)
  bool agg_final = false;  // agg holds the final aggregates (always for the replay kernel, on request for the fast one)
  std::vector<float> planes_h;
  float* planes = nullptr;
  uchar4* guidance = nullptr;
  uint8_t* skip = nullptr;
  uint16_t *start = nullptr, *count = nullptr, *cap = nullptr;
  uint64_t* off = nullptr;
  uint16_t* agg = nullptr;
  uint16_t* agg_pass1 = nullptr;
  uint8_t* raw = nullptr;
  float* depth = nullptr;
  std::vector<DevBuf> bufs;
};

namespace {

int set_err(lux_sgm_ctx* ctx, int code, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->last_error = buf;
  }
  return code;
}

const char* default_message(int code) {
  switch (code) {
    case LUX_ERR_NEAR_FAR: return "The near end has to be smaller than the fard end!";
    case LUX_ERR_NONPOSITIVE: return "Both the near and far end have to be positive!";
    case LUX_ERR_BASELINE: return "Baseline too small, check calibration.";
    case LUX_ERR_SKIPMODE: return "unrecognized sampling pattern";
    case LUX_ERR_BUDGET: return "StereoLayer memory budget exceeded: the BilateralUpsample fallback (mode 0) is not ported";
    case LUX_ERR_UPSAMPLE_SIZE: return "Incorrect output depth size!";
    case LUX_ERR_INDEX: return "Index was outside the bounds of the array (the reference indexes outside an array for these inputs)";
    case LUX_ERR_TIMEOUT: return "a bounded device-side wait timed out";
    case LUX_ERR_ROI: return "invalid ROI requested!";
    case LUX_ERR_EMPTY_IMAGE: return "empty image!";
    default: return "error";
  }
}

#define CK(call)                                                                                                   \
  do {                                                                                                             \
    cudaError_t e_ = (call);                                                                                       \
    if (e_ != cudaSuccess) return set_err(ctx, LUX_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));     \
  } while (0)

// Device allocation from the stream-ordered pool, admitted against the context's HBM budget.
int dev_alloc(lux_sgm_ctx* ctx, std::vector<DevBuf>& owner, size_t bytes, void** out) {
  bytes = (bytes + 255) & ~(size_t)255;
  if (bytes == 0) bytes = 256;
  if (ctx->budget && ctx->in_use + bytes > ctx->budget)
    return set_err(ctx, LUX_ERR_BUDGET, "HBM budget exceeded: %llu bytes in use + %llu requested > %llu budget",
                   (unsigned long long)ctx->in_use, (unsigned long long)bytes, (unsigned long long)ctx->budget);
  void* p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, bytes, ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, LUX_ERR_ALLOC, "device allocation of %llu bytes failed: %s", (unsigned long long)bytes, cudaGetErrorString(e));
  }
  ctx->in_use += bytes;
  owner.push_back({p, bytes});
  *out = p;
  return LUX_OK;
}

void dev_free_all(lux_sgm_ctx* ctx, std::vector<DevBuf>& owner) {
  for (auto& b : owner) {
    cudaFreeAsync(b.p, ctx->stream);
    ctx->in_use -= b.bytes;
  }
  owner.clear();
}

template <class T>
int alloc_t(lux_sgm_ctx* ctx, std::vector<DevBuf>& owner, size_t count, T** out) {
  void* p = nullptr;
  int rc = dev_alloc(ctx, owner, count * sizeof(T), &p);
  *out = static_cast<T*>(p);
  return rc;
}

// Reads and clears the device error word.
int take_device_error(lux_sgm_ctx* ctx) {
  int e = 0;
  CK(cudaMemcpyAsync(&e, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (e) {
    CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    return set_err(ctx, e, "%s", default_message(e));
  }
  return LUX_OK;
}

// Copies an image to the device as a dense RGBA8 buffer (or reuses a dense device image).
int upload_image(lux_sgm_ctx* ctx, std::vector<DevBuf>& owner, const lux_img_rgba8& im, const uint8_t** out) {
  if (!im.data || im.w <= 0 || im.h <= 0 || im.stride < im.w) return set_err(ctx, LUX_ERR_ARG, "invalid image");
  if (im.on_device && im.stride == im.w) {
    *out = im.data;
    return LUX_OK;
  }
  uint8_t* d = nullptr;
  int rc = alloc_t(ctx, owner, (size_t)im.w * im.h * 4, &d);
  if (rc) return rc;
  CK(cudaMemcpy2DAsync(d, (size_t)im.w * 4, im.data, (size_t)im.stride * 4, (size_t)im.w * 4, im.h,
                       im.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
  *out = d;
  return LUX_OK;
}

lux_stereo_params default_params() {
  lux_stereo_params p;
  std::memset(&p, 0, sizeof p);
  p.margin = 1;
  p.plane_density = 2.0f;
  p.scale = 32;
  p.skip_mode = 0;
  p.p1 = 1;
  p.p2scale = 500.0f;
  uint32_t u = 0x3ef6384fu;
  float g;
  std::memcpy(&g, &u, 4);
  p.guidance[0] = g / 6.0f;
  p.guidance[1] = g / 16.0f;
  p.guidance[2] = g / 16.0f;
  p.guidance[3] = 0.0f;
  p.tile = 4;
  return p;
}

struct RangeResult {
  int min_lo, max_hi_raw;
};

// RangeFromPrevious for a layer of size W×H with `planes` against the previous layer (device). start/count: device.
int ranges_from_previous(lux_sgm_ctx* ctx, std::vector<DevBuf>& tmp, const std::vector<float>& planes, const lux_layer* prev, int W,
                         int H, int margin, uint16_t* start, uint16_t* count, RangeResult* rr) {
  std::vector<float> b;
  bool mono = host_range_bounds(planes, b);
  float* db = nullptr;
  int* mm = nullptr;
  void* scratch = nullptr;
  int rc;
  if ((rc = alloc_t(ctx, tmp, b.size(), &db))) return rc;
  if ((rc = alloc_t(ctx, tmp, 2, &mm))) return rc;
  if ((rc = dev_alloc(ctx, tmp, range_from_previous_scratch_bytes(prev->w, prev->h), &scratch))) return rc;
  int init[2] = {INT_MAX, 0};
  CK(cudaMemcpyAsync(db, b.data(), b.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(mm, init, 8, cudaMemcpyHostToDevice, ctx->stream));
  launch_range_from_previous(prev->depth, prev->skip, prev->w, prev->h, db, mono ? 1 : 0, (int)planes.size(), ctx->d_rcp, W, H,
                             margin, start, count, mm, scratch, ctx->stream);
  int res[2];
  CK(cudaMemcpyAsync(res, mm, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  rr->min_lo = res[0];
  rr->max_hi_raw = res[1];
  return LUX_OK;
}

int build_layer(lux_sgm_ctx* ctx, int n_cams, const uint8_t* const* dimg, const int* iw, const int* ih, const uint8_t* gray,
                const lux_calib* calibs, float near_, float far_, const lux_stereo_params& p, int index, int align, const lux_layer* prev,
                int flags, lux_layer* L) {
  int rc;
  if (p.scale <= 0) return set_err(ctx, LUX_ERR_ARG, "scale must be positive");
  if (p.tile < 2) return set_err(ctx, LUX_ERR_UNSUPPORTED, "tile %d: the GPU traversal needs a tile of at least 2", p.tile);
  if (align <= 0) return set_err(ctx, LUX_ERR_ARG, "align must be positive");
  L->ctx = ctx;
  L->index = index;
  L->align = align;
  L->tile = p.tile;
  if ((rc = host_planes(near_, far_, calibs, n_cams, p.plane_density, align, L->planes_h))) return set_err(ctx, rc, "%s", default_message(rc));
  L->n = (int)L->planes_h.size();
  if (n_cams < 2) return set_err(ctx, LUX_ERR_BASELINE, "%s", default_message(LUX_ERR_BASELINE));
  if (n_cams > kMaxCams) return set_err(ctx, LUX_ERR_UNSUPPORTED, "at most %d cameras per layer", kMaxCams);
  L->w = (iw[0] + p.scale - 1) / p.scale;
  L->h = (ih[0] + p.scale - 1) / p.scale;
  const int W = L->w, H = L->h;
  const size_t npx = (size_t)W * H;
  if (p.skip_mode != 0 && p.skip_mode != 2) return set_err(ctx, LUX_ERR_SKIPMODE, "%s", default_message(LUX_ERR_SKIPMODE));
  auto& B = L->bufs;
  if ((rc = alloc_t(ctx, B, (size_t)L->n, &L->planes))) return rc;
  if ((rc = alloc_t(ctx, B, npx, &L->guidance))) return rc;
  if ((rc = alloc_t(ctx, B, npx, &L->skip))) return rc;
  if ((rc = alloc_t(ctx, B, npx, &L->start))) return rc;
  if ((rc = alloc_t(ctx, B, npx, &L->count))) return rc;
  if ((rc = alloc_t(ctx, B, npx, &L->cap))) return rc;
  if ((rc = alloc_t(ctx, B, npx + 1, &L->off))) return rc;
  if ((rc = alloc_t(ctx, B, npx, &L->depth))) return rc;
  cudaStream_t s = ctx->stream;
  CK(cudaMemcpyAsync(L->planes, L->planes_h.data(), (size_t)L->n * 4, cudaMemcpyHostToDevice, s));
  launch_skip_mask(p.skip_mode, W, H, ctx->d_skip_bits, L->skip, s);
  launch_guidance(dimg[0], iw[0], ih[0], W, H, p.scale, L->guidance, s);
  std::vector<DevBuf> tmp;
  struct TmpGuard {
    lux_sgm_ctx* c;
    std::vector<DevBuf>* t;
    ~TmpGuard() { dev_free_all(c, *t); }
  } guard{ctx, &tmp};
  bool uniform = prev == nullptr;
  if (uniform) {  // DenseStereoSgm.cs:43-46
    launch_uniform_ranges(L->start, L->count, L->cap, L->off, (int)npx, L->n, s);
    L->min_lo = 0;
    L->max_hi = ((L->n + align - 1) / align) * align;
    L->volume = (uint64_t)npx * (uint64_t)L->n;
  } else {
    RangeResult rr;
    if ((rc = ranges_from_previous(ctx, tmp, L->planes_h, prev, W, H, p.margin, L->start, L->count, &rr))) return rc;
    L->min_lo = rr.min_lo;
    L->max_hi = ((rr.max_hi_raw + align - 1) / align) * align;
    void* scr = nullptr;
    size_t sb = caps_offsets_scratch_bytes((int)npx);
    if ((rc = dev_alloc(ctx, tmp, sb, &scr))) return rc;
    launch_caps_offsets(L->count, (int)npx, align, L->cap, L->off, scr, sb, s);
    CK(cudaMemcpyAsync(&L->volume, L->off + npx, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    launch_check_caps(L->cap, (int)npx, ctx->d_err, s);
    if ((rc = take_device_error(ctx))) return rc;
  }
  if ((rc = alloc_t(ctx, B, L->volume + 8, &L->agg))) return rc;
  if ((rc = alloc_t(ctx, B, L->volume + 8, &L->raw))) return rc;
  // the fast uniform aggregation writes every aggregate before it reads one; the replay accumulates into zeros
  const bool fast = uniform && !(flags & LUX_LAYER_FORCE_REPLAY) && uniform_fast_supported(W, H, L->n, p.tile, p.p1, p.p2scale);
  if (!fast) CK(cudaMemsetAsync(L->agg, 0, (L->volume + 8) * 2, s));
  if (!uniform) CK(cudaMemsetAsync(L->raw, 0, L->volume + 8, s));
  if (flags & LUX_LAYER_KEEP_PASS1) {
    if ((rc = alloc_t(ctx, B, L->volume + 8, &L->agg_pass1))) return rc;
  }
  LayerGeom g;
  g.W = W; g.H = H; g.n_planes = L->n; g.align = align; g.min_lo = L->min_lo; g.max_hi = L->max_hi; g.tile = p.tile;
  g.planes = L->planes; g.guidance = L->guidance; g.skip = L->skip; g.start = L->start; g.count = L->count; g.cap = L->cap;
  g.off = L->off; g.volume = L->volume; g.uniform = uniform;
  g.timeout_ns = ctx->wait_limit_ns;
  g.stall_block = ctx->stall_block;
  g.never = ctx->d_never;
  // matching cost (DenseStereo.BuildContext + MatchingCost + Normalise)
  CostArgs ca;
  std::memset(&ca, 0, sizeof ca);
  ca.one = 1;
  ca.ref = dimg[0]; ca.rw = iw[0]; ca.rh = ih[0];
  ca.n_others = n_cams - 1;
  for (int k = 1; k < n_cams; k++) {
    ca.other[k - 1] = dimg[k];
    ca.ow[k - 1] = iw[k];
    ca.oh[k - 1] = ih[k];
    host_flow_matrix(calibs[0], calibs[k], ca.warp[k - 1]);
    static const uint16_t wg[4] = {12240, 0, 0, 0}, wc[4] = {8160, 680, 680, 0};
    std::memcpy(ca.wq[k - 1], gray && gray[k] ? wg : wc, sizeof wg);
  }
  {
    uint32_t u = 0x3d17b426u;
    float f;
    std::memcpy(&f, &u, 4);
    volatile float nf = (float)ca.n_others;
    ca.norm = f / nf;
  }
  ca.scale = p.scale;
  // the plane-only projection terms of every camera (DenseStereo.cs:257-259: (z·W2 + W3), one rounding per op)
  std::vector<float> zt_h((size_t)ca.n_others * L->n * 4, 0.0f);
  for (int k = 0; k < ca.n_others; k++)
    for (int i = 0; i < L->n; i++) {
      const float z = L->planes_h[i];
      for (int r = 0; r < 3; r++) {
        volatile float prod = z * ca.warp[k][8 + r];
        zt_h[((size_t)k * L->n + i) * 4 + r] = prod + ca.warp[k][12 + r];
      }
    }
  // An axis-aligned pair (W1 = W2 = W4 = W6 = 0) takes the cost kernel whose 1/pz is per plane: pz is then exactly the
  // plane term, provided it is finite and non-zero for every plane and x·z, y·z stay finite.
  ca.axis = 0;
  if (ca.n_others == 1 && uniform) {
    const float* Wm = ca.warp[0];
    bool ok = Wm[1] == 0.0f && Wm[2] == 0.0f && Wm[4] == 0.0f && Wm[6] == 0.0f;
    double zmax = 0.0;
    for (int i = 0; i < L->n && ok; i++) {
      const float z = L->planes_h[i], pz = zt_h[(size_t)i * 4 + 2];
      ok = std::isfinite(z) && std::isfinite(pz) && pz != 0.0f;
      zmax = std::max(zmax, std::fabs((double)z));
    }
    if (ok && zmax * (double)std::max(iw[0], ih[0]) < 1e37) {
      ca.axis = 1;
      for (int i = 0; i < L->n; i++) {
        volatile float pz = zt_h[(size_t)i * 4 + 2];
        zt_h[(size_t)i * 4 + 3] = 1.0f / pz;  // IEEE division, as __frcp_rn
      }
    }
  }
  float4* zt = nullptr;
  if ((rc = alloc_t(ctx, tmp, zt_h.size() / 4, &zt))) return rc;
  CK(cudaMemcpyAsync(zt, zt_h.data(), zt_h.size() * 4, cudaMemcpyHostToDevice, s));
  // an axis-aligned grey pair at scale 1 with the fast layout: the cost kernel that shares block columns between pixels
  ca.vcols = ca.axis && ca.scale == 1 && cost_all_grey(ca) && uniform && L->n % 8 == 0 && !cost_small_wide_layer(W, H, L->n) ? 1 : 0;
  const size_t phase_words = cost_all_grey(ca) ? 8 : 4;  // per pixel: four phases of {u16 pairs} (grey) or RGBA words
  for (int k = 0; k < ca.n_others; k++) {  // the half-pixel phase images of the other cameras
    uint32_t* ph = nullptr;
    if ((rc = alloc_t(ctx, tmp, phase_words * ca.ow[k] * ca.oh[k], &ph))) return rc;
    ca.phase[k] = ph;
  }
  CK(cudaEventRecord(ctx->ev[0], s));
  launch_phases(ca, s);
  L->cost_kernel = launch_cost(ca, g, zt, L->raw, ctx->d_err, s);
  // aggregation: two passes over the sheared tiles, then WTA
  CK(cudaEventRecord(ctx->ev[1], s));
  const int xsw = 0;  // LUX_SGM_XSW unset: the reference default (DenseStereoSgm.cs:31)
  if (fast) {
    // past 256 planes the fused form is the only fast one: no tuning, and a requested chain or wave form runs fused
    const bool wide = uniform_wide_planes(L->n);
    const int forced = wide ? 1 : (flags & LUX_LAYER_SGM_WAVE) ? 3 : (flags & LUX_LAYER_SGM_SPLIT) ? 2 : (flags & LUX_LAYER_SGM_FUSED) ? 1 : 0;
    int form = forced;
    bool tune = false;
    if (!forced) {
      form = tuned_form(W, H, L->n, p.tile);
      tune = form == 0 && ctx->autotune;
      if (form == 0) form = (size_t)W * H >= 2000000 ? 2 : 1;  // untuned: the path-group chains from about 2 MP
    }
    const int keep = (flags & LUX_LAYER_KEEP_AGG) ? 1 : 0;
    auto scratch_of = [&](int f) {
      return f == 2 ? split_scratch_bytes(W, H, L->n) : f == 3 ? wave_scratch_bytes(W, H, L->n) : uniform_scratch_bytes(W, H, L->n, p.tile);
    };
    auto run_form = [&](int f, void* scr, size_t sb) {
      if (f == 2) return run_sgm_split(g, xsw, p.p1, p.p2scale, p.guidance, L->raw, L->agg, L->agg_pass1, L->depth, keep, scr, sb, ctx->d_err, s);
      if (f == 3) return run_sgm_wave(g, xsw, p.p1, p.p2scale, p.guidance, L->raw, L->agg, L->agg_pass1, L->depth, keep, scr, sb, ctx->d_err, s);
      return run_sgm_uniform(g, xsw, p.p1, p.p2scale, p.guidance, L->raw, L->agg, L->agg_pass1, L->depth, keep, scr, sb, ctx->d_err, s);
    };
    if (tune) {
      // The first solve of this shape times every form on the layer's own volume (the second of two runs) and keeps the
      // fastest for later solves. Each form writes every aggregate and depth it produces and all forms give the same
      // bits, so the layer keeps the last run's results. The reported aggregation time is the chosen form's.
      static const int kForms[3] = {3, 2, 1};
      size_t sb = 0;
      for (int f : kForms) sb = std::max(sb, scratch_of(f));
      void* scr = nullptr;
      if ((rc = dev_alloc(ctx, tmp, sb, &scr))) return rc;
      CK(cudaEventSynchronize(ctx->ev[1]));
      CK(cudaEventElapsedTime(&L->ms_cost, ctx->ev[0], ctx->ev[1]));  // before the timing runs reuse the events
      float best_ms = 0.f;
      int best = 0;
      for (int f : kForms) {
        // an untimed run first: a form's first launch in the process also loads its kernels (lazy module loading) and
        // sets their shared-memory limits, which is not the form's speed
        if ((rc = run_form(f, scr, sb))) return set_err(ctx, LUX_ERR_CUDA, "uniform aggregation launch failed (%d)", rc);
        CK(cudaEventRecord(ctx->ev[1], s));
        if ((rc = run_form(f, scr, sb))) return set_err(ctx, LUX_ERR_CUDA, "uniform aggregation launch failed (%d)", rc);
        CK(cudaEventRecord(ctx->ev[2], s));
        CK(cudaGetLastError());
        if ((rc = take_device_error(ctx))) return rc;
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]));
        if (best == 0 || ms < best_ms) {
          best = f;
          best_ms = ms;
        }
      }
      set_tuned_form(W, H, L->n, p.tile, best);
      L->sgm_kernel = kForms[2];  // the last run's results are in place
      L->agg_final = keep != 0;
      L->ms_sgm = best_ms;
      L->ms_wta = 0.f;
      L->tuned = best;
      return LUX_OK;
    }
    void* scr = nullptr;
    const size_t sb = scratch_of(form);
    if ((rc = dev_alloc(ctx, tmp, sb, &scr))) return rc;
    if ((rc = run_form(form, scr, sb))) return set_err(ctx, LUX_ERR_CUDA, "uniform aggregation launch failed (%d)", rc);
    CK(cudaEventRecord(ctx->ev[2], s));
    CK(cudaEventRecord(ctx->ev[3], s));
    L->sgm_kernel = form;
    L->agg_final = (flags & LUX_LAYER_KEEP_AGG) != 0;
    CK(cudaGetLastError());
    if ((rc = take_device_error(ctx))) return rc;
    CK(cudaEventElapsedTime(&L->ms_cost, ctx->ev[0], ctx->ev[1]));
    CK(cudaEventElapsedTime(&L->ms_sgm, ctx->ev[1], ctx->ev[2]));
    L->ms_wta = 0.f;  // fused into pass -1
    return LUX_OK;
  }
  L->agg_final = true;
  const int bands = (H + p.tile - 1) / p.tile;
  EmuBuffers eb;
  eb.Llen = emu_line_buffer_elems(W, L->max_hi);
  if (eb.Llen > (size_t)INT_MAX - 65536)  // the replay indexes its line buffer with 32-bit integers
    return set_err(ctx, LUX_ERR_UNSUPPORTED, "the exact replay's line buffer of %zu elements is past 32-bit indexing", eb.Llen);
  if ((rc = alloc_t(ctx, tmp, eb.Llen, &eb.L))) return rc;
  if ((rc = alloc_t(ctx, tmp, (size_t)2 * (W + 2) * 4, &eb.Min))) return rc;
  if ((rc = alloc_t(ctx, tmp, (size_t)2 * (W + 2), &eb.RangeS))) return rc;
  if ((rc = alloc_t(ctx, tmp, (size_t)2 * (W + 2), &eb.RangeC))) return rc;
  if ((rc = alloc_t(ctx, tmp, (size_t)2 * (W + 2), &eb.Pix))) return rc;
  if ((rc = alloc_t(ctx, tmp, 2, &eb.ticket))) return rc;
  if ((rc = alloc_t(ctx, tmp, (size_t)2 * bands * kEmuParts, &eb.progress))) return rc;
  emu_init_buffers(eb, W, L->max_hi, align, bands, s);
  launch_sgm_emulate(g, eb, +1, xsw, p.p1, p.p2scale, p.guidance, L->raw, L->agg, ctx->d_err, s);
  if (L->agg_pass1) CK(cudaMemcpyAsync(L->agg_pass1, L->agg, (L->volume + 8) * 2, cudaMemcpyDeviceToDevice, s));
  launch_sgm_emulate(g, eb, -1, xsw, p.p1, p.p2scale, p.guidance, L->raw, L->agg, ctx->d_err, s);
  CK(cudaEventRecord(ctx->ev[2], s));
  launch_wta(g, L->agg, L->depth, ctx->d_err, s);
  CK(cudaEventRecord(ctx->ev[3], s));
  CK(cudaGetLastError());
  if ((rc = take_device_error(ctx))) return rc;
  CK(cudaEventElapsedTime(&L->ms_cost, ctx->ev[0], ctx->ev[1]));
  CK(cudaEventElapsedTime(&L->ms_sgm, ctx->ev[1], ctx->ev[2]));
  CK(cudaEventElapsedTime(&L->ms_wta, ctx->ev[2], ctx->ev[3]));
  return LUX_OK;
}

void destroy_layer(lux_layer* L) {
  if (!L) return;
  if (L->ctx) {
    dev_free_all(L->ctx, L->bufs);
    cudaStreamSynchronize(L->ctx->stream);
  }
  delete L;
}

}  // namespace

extern "C" {

int lux_sgm_create(int device, uint64_t hbm_budget_bytes, lux_sgm_ctx** out) {
  if (!out) return LUX_ERR_ARG;
  *out = nullptr;
  lux_sgm_ctx* ctx = new lux_sgm_ctx();
  ctx->device = device;
  ctx->budget = hbm_budget_bytes;
  auto fail = [&](int code) {
    delete ctx;
    return code;
  };
  if (cudaSetDevice(device) != cudaSuccess) return fail(LUX_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(LUX_ERR_CUDA);
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;  // keep freed blocks in the pool: later requests of the same sizes allocate nothing new
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  if (cudaMalloc(&ctx->d_rcp, 4096 * 4) != cudaSuccess) return fail(LUX_ERR_ALLOC);
  if (cudaMalloc(&ctx->d_err, 2 * sizeof(int)) != cudaSuccess) return fail(LUX_ERR_ALLOC);
  ctx->d_never = ctx->d_err + 1;
  cudaMemcpy(ctx->d_rcp, host_rcp_table(), 4096 * 4, cudaMemcpyHostToDevice);
  {
    uint32_t bits[256];
    host_skip_stream_bits(bits);
    if (cudaMalloc(&ctx->d_skip_bits, sizeof bits) != cudaSuccess) return fail(LUX_ERR_ALLOC);
    cudaMemcpy(ctx->d_skip_bits, bits, sizeof bits, cudaMemcpyHostToDevice);
  }
  {
    std::vector<uint32_t> wt(8192 + 384);
    std::memcpy(wt.data(), host_rsqrt_table(false), 4096 * 4);
    std::memcpy(wt.data() + 4096, host_rsqrt_table(true), 4096 * 4);
    host_lanczos_table(reinterpret_cast<float*>(wt.data() + 8192));
    if (cudaMalloc(&ctx->d_warp, wt.size() * 4) != cudaSuccess) return fail(LUX_ERR_ALLOC);
    cudaMemcpy(ctx->d_warp, wt.data(), wt.size() * 4, cudaMemcpyHostToDevice);
  }
  cudaMemset(ctx->d_err, 0, 2 * sizeof(int));
  for (auto& e : ctx->ev) cudaEventCreate(&e);
  *out = ctx;
  return LUX_OK;
}

void lux_sgm_destroy(lux_sgm_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto& e : ctx->ev) cudaEventDestroy(e);
  cudaFree(ctx->d_rcp);
  cudaFree(ctx->d_skip_bits);
  cudaFree(ctx->d_warp);
  cudaFree(ctx->d_err);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* lux_sgm_last_error(const lux_sgm_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "no context"; }

uint64_t lux_sgm_kernel_launches(void) { return lux::kernel_launches(); }

void* lux_sgm_stream(lux_sgm_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int lux_sgm_pool_high_water(int device, int32_t reset, uint64_t* bytes) {
  if (!bytes) return LUX_ERR_ARG;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) return LUX_ERR_CUDA;
  uint64_t v = 0;
  if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &v) != cudaSuccess) return LUX_ERR_CUDA;
  *bytes = v;
  if (reset) {
    uint64_t zero = 0;
    if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero) != cudaSuccess) return LUX_ERR_CUDA;
  }
  return LUX_OK;
}

int lux_sgm_set_autotune(lux_sgm_ctx* ctx, int32_t on) {
  if (!ctx) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->autotune = on != 0;
  return LUX_OK;
}

int32_t lux_sgm_tuned_form(int32_t w, int32_t h, int32_t n_planes, int32_t tile) { return tuned_form(w, h, n_planes, tile); }

int lux_sgm_set_tuned_form(int32_t w, int32_t h, int32_t n_planes, int32_t tile, int32_t form) {
  if (w <= 0 || h <= 0 || n_planes <= 0 || tile <= 0 || form < 0 || form > 3) return LUX_ERR_ARG;
  set_tuned_form(w, h, n_planes, tile, form);
  return LUX_OK;
}

int lux_sgm_set_wait_limit(lux_sgm_ctx* ctx, uint64_t limit_ns) {
  if (!ctx) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->wait_limit_ns = limit_ns ? limit_ns : kTimeoutNs;
  return LUX_OK;
}

uint64_t lux_sgm_get_wait_limit(const lux_sgm_ctx* ctx) { return ctx ? ctx->wait_limit_ns : 0; }

int lux_sgm_debug_stall(lux_sgm_ctx* ctx, int32_t block) {
  if (!ctx || block < -1 || block == 0) return set_err(ctx, LUX_ERR_ARG, "debug_stall: block must be -1 (off) or >= 1");
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->stall_block = block;
  return LUX_OK;
}

int lux_sgm_revisit_schedule(int32_t w, int32_t h, int32_t tile, int32_t second_pass, int32_t* out, int32_t* y_b) {
  if (w <= 0 || h <= 0 || tile <= 0 || !out) return LUX_ERR_ARG;
  RevisitSchedule sch;
  build_revisit_schedule(w, h, tile, second_pass != 0, sch);
  const std::vector<int>* cols[7] = {&sch.flags, &sch.batch_first, &sch.batch_count, &sch.src0, &sch.src1, &sch.src2, &sch.extra};
  for (int y = 0; y < h; y++)
    for (int k = 0; k < 7; k++) out[(size_t)y * 7 + k] = (*cols[k])[y];
  out[(size_t)h * 7] = sch.end_first;
  out[(size_t)h * 7 + 1] = sch.end_count;
  if (y_b) *y_b = sch.y_b;
  return LUX_OK;
}

int lux_sgm_sync(lux_sgm_ctx* ctx) {
  if (!ctx) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  CK(cudaStreamSynchronize(ctx->stream));
  return LUX_OK;
}

void lux_sgm_default_params(lux_stereo_params* p) {
  if (p) *p = default_params();
}

void lux_sgm_l16_pyramid(lux_stereo_params out[6]) {  // StereoParams.L16Pyramid(false) (DenseStereo.cs:24-30)
  static const int scales[6] = {32, 16, 8, 4, 2, 1}, tiles[6] = {4, 8, 16, 32, 64, 64};
  for (int i = 0; i < 6; i++) {
    out[i] = default_params();
    out[i].scale = scales[i];
    out[i].tile = tiles[i];
    out[i].skip_mode = i >= 4 ? 2 : 0;
    out[i].plane_density = 2.0f;
  }
}

int lux_sgm_planes(float near_, float far_, const lux_calib* calibs, int32_t n_cams, float density, int32_t align, float* out,
                   int32_t* n_out) {
  if (!calibs || !out || !n_out) return LUX_ERR_ARG;
  std::vector<float> pl;
  int rc = host_planes(near_, far_, calibs, n_cams, density, align, pl);
  if (rc) return rc;
  std::memcpy(out, pl.data(), pl.size() * 4);
  *n_out = (int32_t)pl.size();
  return LUX_OK;
}

int lux_sgm_box_filter3(lux_sgm_ctx* ctx, const lux_img_rgba8* src, uint8_t* dst) {
  if (!ctx || !src || !dst) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  std::vector<DevBuf> tmp;
  const uint8_t* d_src = nullptr;
  uint8_t* d_dst = nullptr;
  int rc = upload_image(ctx, tmp, *src, &d_src);
  if (!rc) rc = alloc_t(ctx, tmp, (size_t)src->w * src->h * 4, &d_dst);
  if (!rc) {
    launch_box_filter3(d_src, src->w, src->h, src->w, d_dst, ctx->stream);
    if (cudaMemcpyAsync(dst, d_dst, (size_t)src->w * src->h * 4, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess)
      rc = set_err(ctx, LUX_ERR_CUDA, "box filter copy failed");
  }
  dev_free_all(ctx, tmp);
  return rc;
}

int lux_image_from_grey16(lux_sgm_ctx* ctx, const uint16_t* src, int32_t w, int32_t h, int32_t stride, int32_t src_on_device,
                          int32_t bits, uint8_t* dst) {
  if (!ctx || !src || !dst || w <= 0 || h <= 0 || stride < w || h > 65535 || bits < 9 || bits > 16)
    return set_err(ctx, LUX_ERR_ARG, "image_from_grey16: null pointer, empty size, stride < w, h > 65535 or bits outside 9..16");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  std::vector<DevBuf> tmp;
  const uint16_t* d_src = src;
  int rc = LUX_OK;
  if (!src_on_device) {  // the samples cross as 2 bytes a pixel; the expansion to 4 bytes happens on the GPU
    uint16_t* d = nullptr;
    if ((rc = alloc_t(ctx, tmp, (size_t)w * h, &d))) return rc;
    CK(cudaMemcpy2DAsync(d, (size_t)w * 2, src, (size_t)stride * 2, (size_t)w * 2, h, cudaMemcpyHostToDevice, ctx->stream));
    d_src = d;
  }
  launch_grey16_to_rgba8(d_src, w, h, src_on_device ? stride : w, bits, dst, ctx->stream);
  CK(cudaGetLastError());
  if (!src_on_device) CK(cudaStreamSynchronize(ctx->stream));  // the host buffer may be reused once this returns
  dev_free_all(ctx, tmp);
  return rc;
}

int lux_sgm_layer(lux_sgm_ctx* ctx, int32_t n_cams, const lux_img_rgba8* images, const uint8_t* gray, const lux_calib* calibs,
                  float near_, float far_, const lux_stereo_params* params, int32_t index, int32_t align, const lux_layer* prev,
                  int32_t flags, lux_layer** out) {
  if (!ctx || !images || !calibs || !params || !out || n_cams <= 0) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  *out = nullptr;
  if (n_cams > kMaxCams) return set_err(ctx, LUX_ERR_UNSUPPORTED, "at most %d cameras per layer", kMaxCams);
  lux_layer* L = new lux_layer();
  L->ctx = ctx;
  std::vector<DevBuf> imgs;
  std::vector<const uint8_t*> dimg((size_t)n_cams);
  std::vector<int> iw((size_t)n_cams), ih((size_t)n_cams);
  int rc = LUX_OK;
  for (int k = 0; k < n_cams && !rc; k++) {
    rc = upload_image(ctx, imgs, images[k], &dimg[k]);
    iw[k] = images[k].w;
    ih[k] = images[k].h;
    if (!rc && (flags & LUX_LAYER_PREFILTER)) {  // DenseStereo.BoxFilter3 on the device
      uint8_t* f = nullptr;
      rc = alloc_t(ctx, imgs, (size_t)iw[k] * ih[k] * 4, &f);
      if (!rc) launch_box_filter3(dimg[k], iw[k], ih[k], iw[k], f, ctx->stream);
      dimg[k] = f;
    }
  }
  if (!rc) rc = build_layer(ctx, n_cams, dimg.data(), iw.data(), ih.data(), gray, calibs, near_, far_, *params, index, align, prev,
                            flags, L);
  dev_free_all(ctx, imgs);
  if (rc) {
    destroy_layer(L);
    return rc;
  }
  *out = L;
  return LUX_OK;
}

int lux_sgm_pyramid(lux_sgm_ctx* ctx, int32_t n_cams, const lux_img_rgba8* images, const uint8_t* gray, const lux_calib* calibs,
                    float near_, float far_, int32_t flags, lux_layer* out[6]) {
  if (!ctx || !images || !calibs || !out || n_cams <= 0) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  for (int i = 0; i < 6; i++) out[i] = nullptr;
  if (n_cams > kMaxCams) return set_err(ctx, LUX_ERR_UNSUPPORTED, "at most %d cameras per layer", kMaxCams);
  lux_stereo_params pars[6];
  lux_sgm_l16_pyramid(pars);
  std::vector<DevBuf> imgs;
  std::vector<const uint8_t*> raw_img((size_t)n_cams);
  std::vector<const uint8_t*> filt((size_t)n_cams);
  std::vector<int> iw((size_t)n_cams), ih((size_t)n_cams);
  int rc = LUX_OK;
  for (int k = 0; k < n_cams && !rc; k++) {  // BoxFilter3 per camera, shared by all layers (DenseStereoSgm.cs:335)
    rc = upload_image(ctx, imgs, images[k], &raw_img[k]);
    iw[k] = images[k].w;
    ih[k] = images[k].h;
    uint8_t* f = nullptr;
    if (!rc) rc = alloc_t(ctx, imgs, (size_t)iw[k] * ih[k] * 4, &f);
    if (!rc) launch_box_filter3(raw_img[k], iw[k], ih[k], iw[k], f, ctx->stream);
    filt[k] = f;
  }
  lux_layer* prev = nullptr;
  for (int i = 0; i < 6 && !rc; i++) {
    int align = 8;
    if (prev) {  // align 8 when the estimate fits the 1 GiB budget, else align 2, else unsupported (:340-344)
      int64_t est[2] = {0, 0};
      const int aligns[2] = {8, 2};
      for (int t = 0; t < 2 && !rc; t++) {
        std::vector<float> pl;
        rc = host_planes(near_, far_, calibs, n_cams, pars[i].plane_density, aligns[t], pl);
        if (rc) { set_err(ctx, rc, "%s", default_message(rc)); break; }
        const int W = (iw[0] + pars[i].scale - 1) / pars[i].scale, H = (ih[0] + pars[i].scale - 1) / pars[i].scale;
        const size_t npx = (size_t)W * H;
        std::vector<DevBuf> tmp;
        uint16_t *st = nullptr, *ct = nullptr;
        uint8_t* dsk = nullptr;
        unsigned long long* acc = nullptr;
        RangeResult rr{0, 0};
        if (!rc) rc = alloc_t(ctx, tmp, npx, &st);
        if (!rc) rc = alloc_t(ctx, tmp, npx, &ct);
        if (!rc) rc = alloc_t(ctx, tmp, npx, &dsk);
        if (!rc) rc = alloc_t(ctx, tmp, 1, &acc);
        if (!rc) rc = ranges_from_previous(ctx, tmp, pl, prev, W, H, pars[i].margin, st, ct, &rr);
        unsigned long long cost = 0;
        if (!rc) {
          launch_skip_mask(pars[i].skip_mode, W, H, ctx->d_skip_bits, dsk, ctx->stream);
          cudaMemsetAsync(acc, 0, 8, ctx->stream);
          launch_estimate_terms(ct, dsk, (int)npx, aligns[t], acc, ctx->stream);
          cudaMemcpyAsync(&cost, acc, 8, cudaMemcpyDeviceToHost, ctx->stream);
          if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = set_err(ctx, LUX_ERR_CUDA, "estimate failed");
        }
        dev_free_all(ctx, tmp);
        if (rc) break;
        // MemoryEstimate (DenseStereoSgm.cs:152-155)
        int64_t maxHi = ((rr.max_hi_raw + aligns[t] - 1) / aligns[t]) * aligns[t];
        int64_t w = W, h = H, im = 0;
        for (int k = 0; k < n_cams; k++) im += (int64_t)ih[k] * iw[k] * 4;
        est[t] = (int64_t)cost + w * h * 4 + 20 * (2 * w + 4) + 2 * ((4 * maxHi + 5) * (2 * w + 4) + 8 * w + 16) + im + w * h * 8;
        if (t == 0 && est[0] < 0x40000000LL) break;
      }
      if (rc) break;
      if (est[0] >= 0x40000000LL) {
        if (est[1] >= 0x40000000LL) { rc = set_err(ctx, LUX_ERR_BUDGET, "%s", default_message(LUX_ERR_BUDGET)); break; }
        align = 2;
      }
    }
    lux_layer* L = new lux_layer();
    rc = build_layer(ctx, n_cams, filt.data(), iw.data(), ih.data(), gray, calibs, near_, far_, pars[i], i, align, prev, flags & ~LUX_LAYER_PREFILTER, L);
    if (rc) {
      destroy_layer(L);
      break;
    }
    out[i] = L;
    prev = L;
  }
  dev_free_all(ctx, imgs);
  if (rc) {
    for (int i = 0; i < 6; i++) {
      destroy_layer(out[i]);
      out[i] = nullptr;
    }
  }
  return rc;
}

int lux_layer_get_info(const lux_layer* L, lux_layer_info* info) {
  if (!L || !info) return LUX_ERR_ARG;
  info->w = L->w; info->h = L->h; info->index = L->index; info->align = L->align; info->n_planes = L->n;
  info->min_lo = L->min_lo; info->max_hi = L->max_hi; info->tile = L->tile; info->volume = L->volume;
  info->gpu_ms_cost = L->ms_cost; info->gpu_ms_sgm = L->ms_sgm; info->gpu_ms_wta = L->ms_wta;
  info->sgm_kernel = L->sgm_kernel;
  info->cost_kernel = L->cost_kernel;
  info->tuned = L->tuned;
  return LUX_OK;
}

static const void* field_ptr(const lux_layer* L, int32_t field, size_t* bytes) {
  const size_t npx = (size_t)L->w * L->h;
  switch (field) {
    case LUX_FIELD_DEPTH: *bytes = npx * 4; return L->depth;
    case LUX_FIELD_PLANES: *bytes = (size_t)L->n * 4; return L->planes;
    case LUX_FIELD_SKIP: *bytes = npx; return L->skip;
    case LUX_FIELD_START: *bytes = npx * 2; return L->start;
    case LUX_FIELD_COUNT: *bytes = npx * 2; return L->count;
    case LUX_FIELD_CAP: *bytes = npx * 2; return L->cap;
    case LUX_FIELD_OFFSETS: *bytes = (npx + 1) * 8; return L->off;
    case LUX_FIELD_AGG: *bytes = L->volume * 2; return L->agg_final ? L->agg : nullptr;
    case LUX_FIELD_AGG_PASS1: *bytes = L->volume * 2; return L->agg_pass1;
    case LUX_FIELD_RAW: *bytes = L->volume; return L->raw;
    case LUX_FIELD_GUIDANCE: *bytes = npx * 4; return L->guidance;
    default: *bytes = 0; return nullptr;
  }
}

int lux_layer_read(const lux_layer* L, int32_t field, void* dst, uint64_t bytes) {
  if (!L || !dst) return LUX_ERR_ARG;
  lux_sgm_ctx* ctx = L->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  size_t need = 0;
  const void* p = field_ptr(L, field, &need);
  if (!p) return set_err(ctx, LUX_ERR_ARG, "field %d is not available", field);
  if (bytes != need) return set_err(ctx, LUX_ERR_ARG, "field %d holds %llu bytes, %llu given", field, (unsigned long long)need,
                                    (unsigned long long)bytes);
  CK(cudaMemcpyAsync(dst, p, need, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return LUX_OK;
}

int lux_layer_from_depth(lux_sgm_ctx* ctx, int32_t w, int32_t h, const float* depth, const uint8_t* skip, lux_layer** out) {
  if (!ctx || !depth || !out || w <= 0 || h <= 0) return set_err(ctx, LUX_ERR_ARG, "layer_from_depth: null pointer or empty size");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  lux_layer* L = new lux_layer();
  L->ctx = ctx;
  L->w = w;
  L->h = h;
  L->index = -1;
  const size_t npx = (size_t)w * h;
  int rc;
  if ((rc = alloc_t(ctx, L->bufs, npx, &L->depth)) || (rc = alloc_t(ctx, L->bufs, npx, &L->skip))) {
    destroy_layer(L);
    return rc;
  }
  cudaError_t e = cudaMemcpyAsync(L->depth, depth, npx * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = skip ? cudaMemcpyAsync(L->skip, skip, npx, cudaMemcpyHostToDevice, ctx->stream) : cudaMemsetAsync(L->skip, 0, npx, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    destroy_layer(L);
    return set_err(ctx, LUX_ERR_CUDA, "layer_from_depth: %s", cudaGetErrorString(e));
  }
  *out = L;
  return LUX_OK;
}

const void* lux_layer_device_ptr(const lux_layer* L, int32_t field) {
  if (!L) return nullptr;
  size_t b;
  return field_ptr(L, field, &b);
}

void lux_layer_destroy(lux_layer* L) {
  if (!L) return;
  lux_sgm_ctx* ctx = L->ctx;
  if (ctx) {
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    destroy_layer(L);
  } else {
    delete L;
  }
}

int lux_sgm_upsample(lux_sgm_ctx* ctx, const float* prev_depth, int32_t pw, int32_t ph, int32_t prev_on_device,
                     const lux_img_rgba8* guide, int32_t set_w, int32_t set_h, float sigma, int32_t scale, const float* prev_conf,
                     float* out_depth, float* out_conf) {
  if (!ctx || !prev_depth || !guide || !out_depth || pw <= 0 || ph <= 0) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  std::vector<DevBuf> tmp;
  const int gw = guide->w, gh = guide->h;
  const size_t npo = (size_t)gw * gh, npp = (size_t)pw * ph;
  const uint8_t* dguide = nullptr;
  float *dprev = nullptr, *dout = nullptr, *dconf = nullptr, *dpc = nullptr;
  uint8_t* g2 = nullptr;
  int rc = upload_image(ctx, tmp, *guide, &dguide);
  if (!rc) {
    if (prev_on_device) dprev = const_cast<float*>(prev_depth);
    else if (!(rc = alloc_t(ctx, tmp, npp, &dprev)))
      if (cudaMemcpyAsync(dprev, prev_depth, npp * 4, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) rc = LUX_ERR_CUDA;
  }
  if (!rc) rc = alloc_t(ctx, tmp, npp * 4, &g2);  // RGBA8 at the previous layer's size
  if (!rc) rc = alloc_t(ctx, tmp, npo, &dout);
  const bool conf = prev_conf && out_conf;
  if (!rc && conf) {
    rc = alloc_t(ctx, tmp, npo, &dconf);
    if (!rc) rc = alloc_t(ctx, tmp, npp, &dpc);
    if (!rc && cudaMemcpyAsync(dpc, prev_conf, npp * 4, prev_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                               ctx->stream) != cudaSuccess)
      rc = LUX_ERR_CUDA;
  }
  if (!rc) {
    launch_upsample(dprev, pw, ph, dguide, gw, gh, gw, sigma, ctx->d_rcp, g2, dout, conf ? dpc : nullptr, dconf, ctx->stream);
    if (cudaMemcpyAsync(out_depth, dout, npo * 4, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) rc = LUX_ERR_CUDA;
    if (!rc && conf && cudaMemcpyAsync(out_conf, dconf, npo * 4, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) rc = LUX_ERR_CUDA;
    if (!rc && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = LUX_ERR_CUDA;
    if (rc) set_err(ctx, rc, "upsample failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  dev_free_all(ctx, tmp);
  if (rc) return rc;
  // the size check comes after the computation in the reference too (DenseUpsampleLayer.cs:43)
  if (gw != set_w * scale || gh != set_h * scale) return set_err(ctx, LUX_ERR_UPSAMPLE_SIZE, "%s", default_message(LUX_ERR_UPSAMPLE_SIZE));
  return LUX_OK;
}

}  // extern "C"

// ---------------- depth image cache (DepthCache.cs) ----------------

namespace {

// A device view of a float image: the caller's device pointer, or a copy of host memory owned by `tmp`.
int device_floats(lux_sgm_ctx* ctx, std::vector<DevBuf>& tmp, const float* p, size_t n, int on_device, const float** out) {
  if (on_device) {
    *out = p;
    return LUX_OK;
  }
  float* d = nullptr;
  int rc = alloc_t(ctx, tmp, n, &d);
  if (rc) return rc;
  CK(cudaMemcpyAsync(d, p, n * 4, cudaMemcpyHostToDevice, ctx->stream));
  *out = d;
  return LUX_OK;
}

// Runs `fill` into the caller's output: directly when it is on the device, else through a device buffer copied back.
// Device in, device out: nothing to wait for, the work stays queued on the context's stream. Otherwise the call waits
// for the host copy, or for the work that reads the temporary buffers the caller frees next.
template <class T, class F>
int to_output(lux_sgm_ctx* ctx, std::vector<DevBuf>& tmp, T* out, size_t n, int on_device, F fill) {
  T* d = out;
  int rc = LUX_OK;
  if (!on_device && (rc = alloc_t(ctx, tmp, n, &d))) return rc;
  fill(d);
  CK(cudaGetLastError());
  if (!on_device) CK(cudaMemcpyAsync(out, d, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  if (!on_device || !tmp.empty()) CK(cudaStreamSynchronize(ctx->stream));
  return LUX_OK;
}

}  // namespace

extern "C" int lux_depth_cache_set(lux_sgm_ctx* ctx, const float* depth, int32_t w, int32_t h, int32_t depth_on_device, int32_t cw,
                                   int32_t ch, float* cache, int32_t cache_on_device) {
  if (!ctx) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (cw <= 0 || ch <= 0) return set_err(ctx, LUX_ERR_EMPTY_IMAGE, "%s", default_message(LUX_ERR_EMPTY_IMAGE));  // DepthCache.cs:62
  if (w <= 0 || h <= 0)  // the reference's resample clamps to index -1 of an empty source
    return set_err(ctx, LUX_ERR_INDEX, "depth_cache_set: empty depth map");
  if (!depth || !cache) return set_err(ctx, LUX_ERR_ARG, "depth_cache_set: null pointer");
  cudaSetDevice(ctx->device);
  std::vector<DevBuf> tmp;
  const float* src = nullptr;
  int rc = device_floats(ctx, tmp, depth, (size_t)w * h, depth_on_device, &src);
  if (!rc)
    rc = to_output(ctx, tmp, cache, (size_t)cw * ch, cache_on_device,
                   [&](float* d) { launch_depth_cache_set(src, w, h, cw, ch, ctx->d_rcp, d, ctx->stream); });
  dev_free_all(ctx, tmp);
  return rc;
}

extern "C" int lux_depth_cache_fetch(lux_sgm_ctx* ctx, const float* cache, int32_t cw, int32_t ch, int32_t cache_on_device, int32_t x0,
                                     int32_t y0, int32_t x1, int32_t y1, int32_t dims_w, int32_t dims_h, float* out, int32_t out_on_device) {
  if (!ctx) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  const int rw = x1 - x0, rh = y1 - y0;
  if (rw == 0 || x1 < x0 || rh == 0 || y1 < y0 || (y0 | x0) < 0 || x1 > dims_w || y1 > dims_h)  // DepthCache.cs:163-164
    return set_err(ctx, LUX_ERR_ROI, "%s", default_message(LUX_ERR_ROI));
  if (!cache || !out || cw <= 0 || ch <= 0) return set_err(ctx, LUX_ERR_ARG, "depth_cache_fetch: null pointer or empty cache");
  cudaSetDevice(ctx->device);
  std::vector<DevBuf> tmp;
  const float* img = nullptr;
  int rc = device_floats(ctx, tmp, cache, (size_t)cw * ch, cache_on_device, &img);
  const double sx = (double)cw / dims_w, sy = (double)ch / dims_h;
  if (!rc && sx == 1.0 && sy == 1.0) {  // the plain view of the ROI (:166-172), copied out
    rc = to_output(ctx, tmp, out, (size_t)rw * rh, out_on_device, [&](float* d) {
      cudaMemcpy2DAsync(d, (size_t)rw * 4, img + (size_t)y0 * cw + x0, (size_t)cw * 4, (size_t)rw * 4, rh, cudaMemcpyDeviceToDevice,
                        ctx->stream);
    });
  } else if (!rc) {  // the source window and its offsets (:173-181), in double as the reference
    const int sx0 = std::max((int)std::floor(x0 * sx), 0), sy0 = std::max((int)std::floor(y0 * sy), 0);
    const int sx1 = std::min((int)std::ceil((rw + (double)x0) * sx), (int)cw), sy1 = std::min((int)std::ceil((rh + (double)y0) * sy), (int)ch);
    const double offx = (double)((float)x0 + 0.5f) * sx - sx0, offy = (double)((float)y0 + 0.5f) * sy - sy0;
    const int vw = sx1 <= sx0 || sy1 <= sy0 ? 0 : sx1 - sx0, vh = vw == 0 ? 0 : sy1 - sy0;
    if (vw == 0) rc = set_err(ctx, LUX_ERR_INDEX, "%s", default_message(LUX_ERR_INDEX));
    else
      rc = to_output(ctx, tmp, out, (size_t)rw * rh, out_on_device, [&](float* d) {
        launch_depth_cache_fetch(img, cw, sx0, sy0, vw, vh, offx, offy, sx, sy, rw, rh, ctx->d_rcp, d, ctx->stream);
      });
  }
  dev_free_all(ctx, tmp);
  return rc;
}

// ---------------- stereo-image formation after the ISP, reference guide warp ----------------

namespace {

// The aligned calibration with its lut copied to the device.
int warp_geom(lux_sgm_ctx* ctx, std::vector<DevBuf>& tmp, const lux_aligned_calib* ac, WarpGeom* g) {
  if (!ac || !ac->lut) return set_err(ctx, LUX_ERR_ARG, "aligned calibration without a lut");
  std::memcpy(g->h, ac->H, sizeof g->h);
  g->cx = ac->cx;
  g->cy = ac->cy;
  g->sx = ac->sx;
  g->sy = ac->sy;
  g->neg_zero = -0.0f;
  float* d = nullptr;
  int rc = alloc_t(ctx, tmp, 4096, &d);
  if (rc) return rc;
  CK(cudaMemcpyAsync(d, ac->lut, 4096 * 4, cudaMemcpyHostToDevice, ctx->stream));
  g->lut = d;
  return LUX_OK;
}

const float* warp_taps(const lux_sgm_ctx* ctx) { return reinterpret_cast<const float*>(ctx->d_warp + 8192); }

}  // namespace

extern "C" int lux_warp_f32(lux_sgm_ctx* ctx, const float* src, int32_t sw, int32_t sh, int32_t src_on_device, float gain,
                            const lux_aligned_calib* ac, int32_t dw, int32_t dh, float* dst, int32_t dst_on_device) {
  if (!ctx) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!src || !dst || sw < 1 || sh < 1 || dw < 1 || dh < 1) return set_err(ctx, LUX_ERR_ARG, "warp: null pointer or empty image");
  cudaSetDevice(ctx->device);
  std::vector<DevBuf> tmp;
  WarpGeom g;
  const float* d_src = nullptr;
  int rc = warp_geom(ctx, tmp, ac, &g);
  if (!rc) rc = device_floats(ctx, tmp, src, (size_t)sw * sh * 4, src_on_device, &d_src);
  if (!rc)
    rc = to_output(ctx, tmp, dst, (size_t)dw * dh * 4, dst_on_device, [&](float* d) {
      launch_warp_f32(d_src, sw, sh, gain, g, warp_taps(ctx), ctx->d_warp, dw, dh, nullptr, d, nullptr, ctx->d_err, ctx->stream);
    });
  if (!rc) rc = take_device_error(ctx);
  dev_free_all(ctx, tmp);
  return rc;
}

extern "C" int lux_stereo_image(lux_sgm_ctx* ctx, const float* src, int32_t sw, int32_t sh, int32_t src_on_device, float gain,
                                const lux_aligned_calib* ac, int32_t dw, int32_t dh, int32_t sensor_type, const float* neutral,
                                uint8_t* out_rgba8, int32_t out_on_device, float* out_yuv, int32_t yuv_on_device) {
  if (!ctx) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!src || !out_rgba8 || !neutral || sw < 1 || sh < 1 || dw < 1 || dh < 1)
    return set_err(ctx, LUX_ERR_ARG, "stereo image: null pointer or empty image");
  cudaSetDevice(ctx->device);
  std::vector<DevBuf> tmp;
  WarpGeom g;
  YuvRows m;
  host_yuv_matrix(sensor_type, neutral, &m.m[0][0]);
  const float* d_src = nullptr;
  float* d_yuv = out_yuv && yuv_on_device ? out_yuv : nullptr;
  const size_t npx = (size_t)dw * dh;
  int rc = warp_geom(ctx, tmp, ac, &g);
  if (!rc) rc = device_floats(ctx, tmp, src, (size_t)sw * sh * 4, src_on_device, &d_src);
  if (!rc && out_yuv && !yuv_on_device) rc = alloc_t(ctx, tmp, npx * 4, &d_yuv);
  if (!rc)
    rc = to_output(ctx, tmp, out_rgba8, npx * 4, out_on_device, [&](uint8_t* d) {
      launch_warp_f32(d_src, sw, sh, gain, g, warp_taps(ctx), ctx->d_warp, dw, dh, &m, d_yuv, d, ctx->d_err, ctx->stream);
    });
  if (!rc && out_yuv && !yuv_on_device) {
    CK(cudaMemcpyAsync(out_yuv, d_yuv, npx * 16, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  if (!rc) rc = take_device_error(ctx);
  dev_free_all(ctx, tmp);
  return rc;
}

extern "C" int lux_stereo_image_transfer(lux_sgm_ctx* ctx, const float* src, int32_t sw, int32_t sh, int32_t src_on_device,
                                         float gain, const lux_aligned_calib* ac, int32_t dw, int32_t dh, int32_t sensor_type,
                                         const float* neutral, const float* ref_yuv, int32_t ref_on_device, const lux_calib* ref_view,
                                         const lux_calib* view, uint8_t* out_rgba8, int32_t out_on_device, float* out_F) {
  if (!ctx) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ref_yuv || !ref_view) return set_err(ctx, LUX_ERR_ARG, "Empty reference yuv.");  // StereoImageBuilder.cs:73
  if (!src || !out_rgba8 || !neutral || !view || sw < 1 || sh < 1 || dw < 1 || dh < 1)
    return set_err(ctx, LUX_ERR_ARG, "stereo image: null pointer or empty image");
  cudaSetDevice(ctx->device);
  std::vector<DevBuf> tmp;
  WarpGeom g;
  YuvRows m;
  host_yuv_matrix(sensor_type, neutral, &m.m[0][0]);
  const size_t npx = (size_t)dw * dh;
  const float* d_src = nullptr;
  float* d_yuv = nullptr;
  uint8_t* d_out = out_on_device ? out_rgba8 : nullptr;
  int rc = warp_geom(ctx, tmp, ac, &g);
  if (!rc) rc = device_floats(ctx, tmp, src, (size_t)sw * sh * 4, src_on_device, &d_src);
  if (!rc) rc = alloc_t(ctx, tmp, npx * 4, &d_yuv);
  if (!rc && !d_out) rc = alloc_t(ctx, tmp, npx * 4, &d_out);
  if (rc) {
    dev_free_all(ctx, tmp);
    return rc;
  }
  // the warped YUV image on the device, then its statistics and the reference crop's on the host (a serial recurrence)
  launch_warp_f32(d_src, sw, sh, gain, g, warp_taps(ctx), ctx->d_warp, dw, dh, &m, d_yuv, d_out, ctx->d_err, ctx->stream);
  std::vector<float> work(npx * 4), ref_h;
  CK(cudaMemcpyAsync(work.data(), d_yuv, npx * 16, cudaMemcpyDeviceToHost, ctx->stream));
  const float* ref = ref_yuv;
  if (ref_on_device) {
    ref_h.resize(npx * 4);
    CK(cudaMemcpyAsync(ref_h.data(), ref_yuv, npx * 16, cudaMemcpyDeviceToHost, ctx->stream));
    ref = ref_h.data();
  }
  CK(cudaStreamSynchronize(ctx->stream));
  rc = take_device_error(ctx);
  if (!rc) {
    int rect[4];
    host_crop_rect(*ref_view, *view, dw, dh, rect);  // StereoColorTransfer.Transfer (StereoColorTransfer.cs:128-138)
    const int X0 = std::max(0, rect[0]), Y0 = std::max(0, rect[1]), X1 = std::min((int)dw, rect[2]), Y1 = std::min((int)dh, rect[3]);
    const ColourStats sw_ = host_colour_stats(work.data(), dw, dh, dw, 0);
    ColourStats sr{};
    if (X1 - X0 > 0 && Y1 - Y0 > 0) sr = host_colour_stats(ref, X1 - X0, Y1 - Y0, dw, (size_t)Y0 * dw + X0);
    ColourF F;
    host_colour_solve(sw_, sr, F.f);
    if (out_F) std::memcpy(out_F, F.f, sizeof F.f);
    launch_colour_apply(d_yuv, (int)npx, F, d_out, ctx->stream);
    CK(cudaGetLastError());
    if (!out_on_device) CK(cudaMemcpyAsync(out_rgba8, d_out, npx * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  dev_free_all(ctx, tmp);
  return rc;
}

namespace {

// The census mode over n pairs (the reference image against others[0..n)) on the context's stream: per pair device
// buffers in tmp, disparities in pairs.p[k].disp. Validates the arguments as the public calls document.
int census_batch(lux_sgm_ctx* ctx, std::vector<DevBuf>& tmp, int n, const lux_img_rgba8& ref, const lux_img_rgba8* others,
                 const int32_t* Ds, uint32_t p1, uint32_t p2, int subpixel, int lr, int max_diff, CensusPairs& pairs) {
  if (n < 1 || n > kMaxFusePairs) return set_err(ctx, LUX_ERR_ARG, "census: 1 to 16 pairs");
  if (p2 > 8129 || p1 > 8129) return set_err(ctx, LUX_ERR_ARG, "census: P1/P2 too large, path sums would pass 16 bits");
  for (int k = 0; k < n; k++) {
    if (others[k].w != ref.w || others[k].h != ref.h) return set_err(ctx, LUX_ERR_ARG, "census: the two images differ in size");
    if (Ds[k] < 1 || Ds[k] > 256) return set_err(ctx, LUX_ERR_ARG, "census: max_disparity must be 1..256");
  }
  const int w = ref.w, h = ref.h;
  const size_t npx = (size_t)w * h;
  const uint8_t* d_ref = nullptr;
  std::vector<const uint8_t*> d_oth(n);
  uint64_t* cl = nullptr;
  int rc = upload_image(ctx, tmp, ref, &d_ref);
  if (!rc) rc = alloc_t(ctx, tmp, npx, &cl);
  for (int k = 0; k < n && !rc; k++) {
    CensusPair& pr = pairs.p[k];
    pr.D = Ds[k];
    const size_t Dp = 32 * (size_t)census_lpt(Ds[k]);
    if (!rc) rc = upload_image(ctx, tmp, others[k], &d_oth[k]);
    if (!rc) rc = alloc_t(ctx, tmp, npx, &pr.cr);
    if (!rc) rc = alloc_t(ctx, tmp, npx * Dp, &pr.cost);
    if (!rc) rc = alloc_t(ctx, tmp, npx * Dp, &pr.S);
    if (!rc) rc = alloc_t(ctx, tmp, npx, &pr.dl);
    if (!rc) rc = alloc_t(ctx, tmp, npx, &pr.dr);
    if (!rc) rc = alloc_t(ctx, tmp, npx, &pr.disp);
  }
  if (rc) return rc;
  launch_census_batch(d_ref, d_oth.data(), n, w, h, w, 4, p1, p2, subpixel, lr, max_diff, cl, pairs, ctx->stream);
  CK(cudaGetLastError());
  return LUX_OK;
}

}  // namespace

extern "C" int lux_census_sgm(lux_sgm_ctx* ctx, const lux_img_rgba8* left, const lux_img_rgba8* right, const lux_census_params* p,
                              float* out_disp, int32_t out_on_device) {
  if (!ctx) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!left || !right || !p || !out_disp) return set_err(ctx, LUX_ERR_ARG, "census: null pointer");
  cudaSetDevice(ctx->device);
  std::vector<DevBuf> tmp;
  CensusPairs pairs{};
  const int32_t D = p->max_disparity;
  int rc = census_batch(ctx, tmp, 1, *left, right, &D, p->p1, p->p2, p->subpixel, p->lr_check, p->lr_max_diff, pairs);
  const size_t npx = (size_t)left->w * left->h;
  if (!rc) {
    CK(cudaMemcpyAsync(out_disp, pairs.p[0].disp, npx * 4, out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  dev_free_all(ctx, tmp);
  return rc;
}

extern "C" int lux_census_capture(lux_sgm_ctx* ctx, int32_t n, const lux_img_rgba8* ref, const lux_img_rgba8* others,
                                  const int32_t* max_disparity, const float* fb, const lux_census_params* p, float* out_depth,
                                  int32_t out_on_device, float* out_disps) {
  if (!ctx) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ref || !others || !max_disparity || !fb || !p || !out_depth) return set_err(ctx, LUX_ERR_ARG, "census capture: null pointer");
  cudaSetDevice(ctx->device);
  std::vector<DevBuf> tmp;
  CensusPairs pairs{};
  int rc = census_batch(ctx, tmp, n, *ref, others, max_disparity, p->p1, p->p2, p->subpixel, p->lr_check, p->lr_max_diff, pairs);
  const size_t npx = (size_t)ref->w * ref->h;
  const float** d_list = nullptr;
  float* d_fb = nullptr;
  if (!rc) rc = alloc_t(ctx, tmp, (size_t)n, &d_list);
  if (!rc) rc = alloc_t(ctx, tmp, (size_t)n, &d_fb);
  if (!rc) {
    std::vector<const float*> lst(n);
    for (int k = 0; k < n; k++) lst[k] = pairs.p[k].disp;
    CK(cudaMemcpyAsync(d_list, lst.data(), n * sizeof(float*), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_fb, fb, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    rc = to_output(ctx, tmp, out_depth, npx, out_on_device, [&](float* d) { launch_fuse(d_list, d_fb, n, (int)npx, d, ctx->stream); });
    if (!rc && out_disps)
      for (int k = 0; k < n; k++)
        CK(cudaMemcpyAsync(out_disps + (size_t)k * npx, pairs.p[k].disp, npx * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  dev_free_all(ctx, tmp);
  return rc;
}

extern "C" int lux_fuse_disparities(lux_sgm_ctx* ctx, const float* const* disps, const float* fb, int32_t n, int32_t w, int32_t h,
                                    int32_t on_device, float* out_depth, int32_t out_on_device) {
  if (!ctx) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!disps || !fb || !out_depth || n < 1 || n > kMaxFusePairs || w < 1 || h < 1)
    return set_err(ctx, LUX_ERR_ARG, "fuse: null pointer, bad size or more than 16 pairs");
  cudaSetDevice(ctx->device);
  const size_t npx = (size_t)w * h;
  std::vector<DevBuf> tmp;
  std::vector<const float*> dptr(n);
  int rc = LUX_OK;
  for (int k = 0; k < n && !rc; k++) rc = device_floats(ctx, tmp, disps[k], npx, on_device, &dptr[k]);
  const float** d_list = nullptr;
  float* d_fb = nullptr;
  if (!rc) rc = alloc_t(ctx, tmp, (size_t)n, &d_list);
  if (!rc) rc = alloc_t(ctx, tmp, (size_t)n, &d_fb);
  if (!rc) {
    CK(cudaMemcpyAsync(d_list, dptr.data(), n * sizeof(float*), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_fb, fb, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    rc = to_output(ctx, tmp, out_depth, npx, out_on_device, [&](float* d) { launch_fuse(d_list, d_fb, n, (int)npx, d, ctx->stream); });
  }
  if (!rc) CK(cudaStreamSynchronize(ctx->stream));
  dev_free_all(ctx, tmp);
  return rc;
}

extern "C" int lux_warp_rgba8(lux_sgm_ctx* ctx, const lux_img_rgba8* src, const lux_aligned_calib* ac, int32_t dw, int32_t dh,
                              uint8_t* dst, int32_t dst_on_device) {
  if (!ctx) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!src || !dst || dw < 1 || dh < 1) return set_err(ctx, LUX_ERR_ARG, "warp: null pointer or empty destination");
  if (src->w < 1 || src->h < 1) return set_err(ctx, LUX_ERR_ARG, "empty source image!");  // ReferenceGuide.cs:110
  cudaSetDevice(ctx->device);
  std::vector<DevBuf> tmp;
  WarpGeom g;
  const uint8_t* d_src = nullptr;
  int rc = warp_geom(ctx, tmp, ac, &g);
  if (!rc) rc = upload_image(ctx, tmp, *src, &d_src);
  if (!rc)
    rc = to_output(ctx, tmp, dst, (size_t)dw * dh * 4, dst_on_device, [&](uint8_t* d) {
      launch_warp_rgba8(d_src, src->w, src->h, src->w, g, warp_taps(ctx), ctx->d_warp, dw, dh, d, ctx->d_err, ctx->stream);
    });
  if (!rc) rc = take_device_error(ctx);
  dev_free_all(ctx, tmp);
  return rc;
}

extern "C" void lux_lanczos_table(float* out384) {
  if (out384) host_lanczos_table(out384);
}

extern "C" void lux_yuv_matrix(int32_t sensor_type, const float* neutral, float* out12) {
  if (neutral && out12) host_yuv_matrix(sensor_type, neutral, out12);
}

// ---------------- allocation-free upsample ----------------
namespace {

// The resampled guidance (RGBA8 at the previous layer's size) of lux_sgm_upsample_noalloc lives in module-static device
// memory, so that call allocates nothing: it serves hosts whose GPU memory belongs to another allocator, or whose
// request loop must not synchronise on cudaMalloc / cudaFree. Every GPU that loads the library holds these 16 MiB until
// exit. Every byte the bilateral pass reads is written earlier in the same call (k_shift_resize covers all pw·ph
// pixels), so nothing has to start at zero. Host code must not pass the array's name to a kernel (on the host it is
// only a stand-in for the symbol): upsample_scratch() looks up its device address.
constexpr size_t kNoAllocMaxPixels = LUX_UPSAMPLE_NOALLOC_MAX_PIXELS;
static __device__ __align__(256) uint8_t g_upsample_scratch[kNoAllocMaxPixels * 4];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// The array's address on `device`, looked up once per device; the caller has made `device` current.
int upsample_scratch(int device, uint8_t** out) {
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (device < 0 || device >= kMaxDevices) return LUX_ERR_ARG;
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_upsample_scratch) != cudaSuccess || !p) return LUX_ERR_CUDA;
    g_scratch_ptr[device] = p;
  }
  *out = static_cast<uint8_t*>(g_scratch_ptr[device]);
  return LUX_OK;
}

}  // namespace

extern "C" int lux_sgm_upsample_noalloc(lux_sgm_ctx* ctx, const float* prev_depth, int32_t pw, int32_t ph, const lux_img_rgba8* guide,
                                        int32_t set_w, int32_t set_h, float sigma, int32_t scale, const float* prev_conf,
                                        float* out_depth, float* out_conf) {
  if (!ctx) return LUX_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!prev_depth || !guide || !out_depth || pw <= 0 || ph <= 0)
    return set_err(ctx, LUX_ERR_ARG, "upsample_noalloc: null pointer or non-positive previous size");
  if (!guide->data || !guide->on_device || guide->w <= 0 || guide->h <= 0 || guide->stride < guide->w)
    return set_err(ctx, LUX_ERR_ARG, "upsample_noalloc: the guide must be a device image (on_device != 0, w, h > 0, stride >= w)");
  const unsigned long long npp = (unsigned long long)pw * (unsigned long long)ph;
  if (npp > kNoAllocMaxPixels)
    return set_err(ctx, LUX_ERR_ARG, "upsample_noalloc: pw*ph = %llu exceeds the static scratch of %llu pixels", npp,
                   (unsigned long long)kNoAllocMaxPixels);
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, LUX_ERR_CUDA, "upsample_noalloc: cudaSetDevice failed");
  uint8_t* g2 = nullptr;
  int rc = upsample_scratch(ctx->device, &g2);
  if (rc) return set_err(ctx, rc, "upsample_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(cudaGetLastError()));
  const bool conf = prev_conf && out_conf;
  launch_upsample(prev_depth, pw, ph, guide->data, guide->w, guide->h, guide->stride, sigma, ctx->d_rcp, g2, out_depth,
                  conf ? prev_conf : nullptr, conf ? out_conf : nullptr, ctx->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return set_err(ctx, LUX_ERR_CUDA, "upsample_noalloc failed: %s", cudaGetErrorString(e));
  // the size check comes after the computation in the reference too (DenseUpsampleLayer.cs:43)
  if (guide->w != set_w * scale || guide->h != set_h * scale)
    return set_err(ctx, LUX_ERR_UPSAMPLE_SIZE, "%s", default_message(LUX_ERR_UPSAMPLE_SIZE));
  return LUX_OK;
}
