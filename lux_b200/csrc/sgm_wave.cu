// Fused four-path wavefront aggregation of a uniform layer, lean form (bit-exact with DenseStereoSgm.cs:181-324 through
// revisit_schedule.h, like k_sgm_uniform, whose schedule it keeps).
//
// Shape: a block owns kWRows consecutive rows of a pass (mirrored coordinates in pass -1), one warp per row, plus a
// loader warp (the row above the block, from the global band buffer of the block above) and a publisher warp (the
// block's last row out to its own band buffer). Row y takes pixel x once row y-1 has finished x+1, so the rows run as a
// wavefront; the four paths of a pixel are fused, so each pass reads the raw volume once and touches the aggregates once
// (pass +1 writes them, pass -1 reads them and takes the WTA): 6 bytes per DE over both passes.
//
// What makes it lean, per pixel of a row (LPT planes a lane as LPT/2 packed u16 pairs):
//   * the hand-over is a progress counter per row in shared memory (a CTA-scope release store after the ring slot is
//     written, acquire loads by the neighbours), checked against a cached value first, so a row that is far enough
//     behind the row above reads no counter at all; the row above checks the row below the same way before it reuses a
//     ring slot;
//   * ring slots are read and written as 16-byte vectors, the three path minima of a slot as one 16-byte record;
//   * every path minimum is carried duplicated in both u16 halves (min(v, swap(v)) before the warp's redux.min), which is
//     the form the recurrence subtracts and the P2 term adds, so no per-path unpacking is needed;
//   * the d-1 / d+1 neighbours of a lane's pairs come from one byte permute per pair (the pair of planes 2i+1, 2i+2 is
//     both the d+1 word of pair i and the d-1 word of pair i+1), and the aggregate takes the four paths with two
//     three-input adds per word.
// Exactness without saturation is as in k_sgm_uniform: with P2 <= 1744 every stored L is below 2000 (a never-written
// word), every candidate of the minimum is at least the previous minimum, and 16 contributions never exceed 65535.
#include <cstring>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "revisit_schedule.h"
#include "sgm_paths.cuh"

namespace lux {

namespace {

constexpr int kWRows = 16;             // rows of the recurrence per block (one warp each)
constexpr int kWWarps = kWRows + 2;    // plus the loader and the publisher
constexpr int kWRing = 8;              // ring slots (pixels) per row
constexpr int kWBandBufs = 4;          // band buffers in rotation
constexpr int kWPublish = 4;           // the publisher releases the global band progress every kWPublish pixels
constexpr int kWLoad = 4;              // pixels the loader brings in at once

LUX_DEV uint32_t swap16(uint32_t v) { return __byte_perm(v, 0, 0x1032); }
// Minimum over the warp of a lane's packed pairs, duplicated in both halves.
template <int LPT>
LUX_DEV uint32_t warp_min_dup(const V<LPT>& v) {
  uint32_t m = v.r[0];
#pragma unroll
  for (int i = 1; i < LPT / 2; i++) m = vmin2(m, v.r[i]);
  m = vmin2(m, swap16(m));
  return __reduce_min_sync(0xffffffffu, m);
}

// Vector loads and stores of a lane's planes in shared memory (16, 8 or 4 bytes).
template <int LPT>
LUX_DEV void sload(V<LPT>& v, const uint16_t* base, int lane) {
  if constexpr (LPT == 8) {
    const uint4 t = reinterpret_cast<const uint4*>(base)[lane];
    v.r[0] = t.x; v.r[1] = t.y; v.r[2] = t.z; v.r[3] = t.w;
  } else if constexpr (LPT == 4) {
    const uint2 t = reinterpret_cast<const uint2*>(base)[lane];
    v.r[0] = t.x; v.r[1] = t.y;
  } else {
    v.r[0] = reinterpret_cast<const uint32_t*>(base)[lane];
  }
}
template <int LPT>
LUX_DEV void sstore(const V<LPT>& v, uint16_t* base, int lane) {
  if constexpr (LPT == 8) reinterpret_cast<uint4*>(base)[lane] = make_uint4(v.r[0], v.r[1], v.r[2], v.r[3]);
  else if constexpr (LPT == 4) reinterpret_cast<uint2*>(base)[lane] = make_uint2(v.r[0], v.r[1]);
  else reinterpret_cast<uint32_t*>(base)[lane] = v.r[0];
}

// The four paths of one pixel (DenseStereoSgm.cs:276-313). nb[p]: the path-p neighbour's L, md[p]: its minimum in both
// halves; p2w: the pixel's P2 of paths 0, 1 (word x) and 2, 3 (word y). Returns the new L of each path and its minimum
// (both halves), and adds the four paths to acc.
template <int LPT, bool FULL>
LUX_DEV void wave_paths(const V<LPT> (&nb)[4], const uint32_t (&md)[4], uint2 p2w, uint32_t p1x2, const V<LPT>& raw2, bool active,
                        int lane, V<LPT> (&out)[4], V<LPT>& acc, uint32_t (&mdo)[4]) {
  constexpr int NR = LPT / 2;
  const uint32_t p2d[4] = {dup16(p2w.x), __byte_perm(p2w.x, 0, 0x3232), dup16(p2w.y), __byte_perm(p2w.y, 0, 0x3232)};
  uint32_t prev[4], next[4];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    prev[p] = __shfl_up_sync(0xffffffffu, nb[p].r[NR - 1], 1);
    next[p] = __shfl_down_sync(0xffffffffu, nb[p].r[0], 1);
  }
#pragma unroll
  for (int p = 0; p < 4; p++) {
    if (lane == 0) prev[p] = kInit2;   // plane -1: 2000
    if (lane == 31) next[p] = kInit2;  // plane n (or a padding lane): 2000
    const uint32_t p2x = p2d[p] + md[p];  // P2 + minPrev <= 3744 in each half: no carry between the halves
    // u[i + 1] = (L[2i+1], L[2i+2]): the d+1 word of pair i and the d-1 word of pair i+1
    uint32_t u[NR + 1];
    u[0] = pair_of(prev[p], nb[p].r[0]);
#pragma unroll
    for (int i = 0; i + 1 < NR; i++) u[i + 1] = pair_of(nb[p].r[i], nb[p].r[i + 1]);
    u[NR] = pair_of(nb[p].r[NR - 1], next[p]);
#pragma unroll
    for (int i = 0; i < NR; i++) {
      uint32_t t = vmin2(u[i], u[i + 1]) + p1x2;          // min(L[d-1], L[d+1]) + P1
      t = vmin2(vmin2(t, nb[p].r[i]), p2x);               // with L[d] and P2 + minPrev
      uint32_t lc = t + raw2.r[i] - md[p];                 // raw + m - minPrev, each half in [0, 2000)
      if (!FULL) lc = active ? lc : kInit2;                // padding lanes keep 2000
      out[p].r[i] = lc;
    }
    mdo[p] = warp_min_dup<LPT>(out[p]);
  }
#pragma unroll
  for (int i = 0; i < NR; i++) acc.r[i] = acc.r[i] + out[0].r[i] + out[1].r[i] + (out[2].r[i] + out[3].r[i]);
}

// Bounded wait until *p >= target (a CTA-scope acquire), `seen` caching the last value read. Gives up when *stop is set
// or after timeout_ns (then error 11 and *stop).
LUX_DEV bool wait_prog(const int* p, int target, int& seen, volatile int* stop, int* err, uint64_t timeout_ns) {
  if (seen >= target) return true;
  seen = ld_acquire_cta(p);
  if (seen >= target) return true;
  const uint64_t t0 = global_ns();
  for (unsigned it = 0;; it++) {
    __nanosleep(16);
    seen = ld_acquire_cta(p);
    if (seen >= target) return true;
    if ((it & 15) == 15) {
      if (*stop) return false;
      if (global_ns() - t0 > timeout_ns) {
        atomicCAS(err, 0, 11);
        *stop = 1;
        return false;
      }
    }
  }
}

struct WaveArgs {
  UniArgs u;
  uint16_t* bnd;   // [kWBandBufs][W][3][Dp]
  uint4* bnd_md;   // [kWBandBufs][W] path minima (both halves) of paths 1, 2, 3
};

template <int LPT>
constexpr size_t wave_smem_bytes() {
  return (size_t)(kWRows + 1) * kWRing * 3 * Dp_of(LPT) * 2 + (size_t)(kWRows + 1) * kWRing * 16;
}

template <int LPT, bool FULL, bool PASS2, bool MB>
__global__ void __launch_bounds__(kWWarps * 32, 1) k_wave(const WaveArgs wa) {
  constexpr int NR = LPT / 2, Dp = Dp_of(LPT);
  const UniArgs& a = wa.u;
  extern __shared__ __align__(16) uint16_t smem_wave[];
  auto vec = [&](int set, int slot, int p) { return smem_wave + (((size_t)set * kWRing + slot) * 3 + p) * Dp; };
  uint4* mins = reinterpret_cast<uint4*>(smem_wave + (size_t)(kWRows + 1) * kWRing * 3 * Dp);
  auto mrec = [&](int set, int slot) -> uint4& { return mins[set * kWRing + slot]; };
  // prog[r]: pixels finished by row r (r < kWRows), loaded by the loader (kWRows), copied out by the publisher (kWRows+1)
  __shared__ int prog[kWRows + 2];
  // MB: the hand-over in is a full mbarrier per ring slot (the waiting warp is suspended by the hardware instead of
  // polling the counter); the counters then serve only the check that a slot is free again
  __shared__ uint64_t full_bar[MB ? (kWRows + 1) * kWRing : 1];
  __shared__ int s_cb;
  __shared__ volatile int s_stop;
  __shared__ float s_planes[256];  // the WTA's plane depths (pass -1)
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (PASS2)
    for (int i = tid; i < a.n; i += blockDim.x) s_planes[i] = a.planes[i];
  if (tid < kWRows + 2) prog[tid] = 0;
  if (MB && tid < (kWRows + 1) * kWRing) mbar_init(&full_bar[tid], 1);
  if (tid == 0) {
    s_cb = atomicAdd(a.ticket, 1);
    s_stop = 0;
  }
  __syncthreads();
  const int cb = s_cb;
  const int y0 = cb * kWRows;
  const int rows = min(kWRows, a.H - y0);  // rows of this block inside the image
  const bool below_exists = y0 + kWRows < a.H;
  const bool active = FULL || lane * LPT < a.n;
  const int W = a.W, c = W - 1;
  const uint16_t* bnd_up = wa.bnd + (size_t)((cb + kWBandBufs - 1) % kWBandBufs) * W * 3 * Dp;
  const uint4* bnd_up_md = wa.bnd_md + (size_t)((cb + kWBandBufs - 1) % kWBandBufs) * W;
  uint16_t* bnd_me = wa.bnd + (size_t)(cb % kWBandBufs) * W * 3 * Dp;
  uint4* bnd_me_md = wa.bnd_md + (size_t)(cb % kWBandBufs) * W;
  auto wait = [&](int idx, int target, int& seen) { return wait_prog(&prog[idx], target, seen, &s_stop, a.err, a.timeout_ns); };
  // MB: pixel p of set `set` is in its ring slot (phase p / kWRing of the slot's full barrier)
  auto wait_full = [&](int set, int p) {
    return mbar_wait(&full_bar[set * kWRing + (p & (kWRing - 1))], (uint32_t)(p / kWRing) & 1u, &s_stop, a.err, a.timeout_ns);
  };

  if (w == kWRows) {
    // ---------------- loader: the row above the block into set kWRows ----------------
    if (y0 >= a.H) return;
    int avail = cb > 0 ? 0 : W, cons = 0;
    const int* gprog = cb == a.stall_block ? a.never : a.progress + (cb - 1);
    for (int xb = 0; xb < W && !s_stop; xb += kWLoad) {
      const int xe = min(W, xb + kWLoad);
      // row 0 is done with the slots of pixels xe-1-kWRing and before: it finished pixel xe-kWRing (>= x-kWRing+2)
      if (!wait(0, xe - kWRing + 1, cons)) break;
      if (avail < xe) {
        int v = 0;
        if (lane == 0) v = wait_at_least_value(gprog, xe, a.err, 11, a.timeout_ns);
        v = __shfl_sync(0xffffffffu, v, 0);
        __syncwarp();  // lane 0's acquire orders the band-buffer reads of every lane
        if (v < 0) {
          s_stop = 1;
          break;
        }
        avail = v;
      }
      V<LPT> L[kWLoad][3];
      uint4 md[kWLoad];
#pragma unroll
      for (int k = 0; k < kWLoad; k++) {
        const int x = xb + k;
        if (x >= xe) break;
        if (cb > 0) {
#pragma unroll
          for (int p = 0; p < 3; p++) vload<LPT>(L[k][p], bnd_up + ((size_t)x * 3 + p) * Dp, lane);
          md[k] = __ldcg(bnd_up_md + x);
        } else {
          uint32_t m[3];
#pragma unroll
          for (int p = 1; p < 4; p++) {
            Src<LPT> s;
            if (a.edge_read) src_edge<LPT>(a, s, a.dir > 0 ? x : W - 1 - x, p, lane);
            else src_init(s);
            L[k][p - 1] = s.L;
            m[p - 1] = dup16(s.mn);
          }
          md[k] = make_uint4(m[0], m[1], m[2], 0u);
        }
      }
#pragma unroll
      for (int k = 0; k < kWLoad; k++) {
        const int x = xb + k;
        if (x >= xe) break;
        const int sl = x & (kWRing - 1);
#pragma unroll
        for (int p = 0; p < 3; p++) sstore<LPT>(L[k][p], vec(kWRows, sl, p), lane);
        if (lane == 0) mrec(kWRows, sl) = md[k];
      }
      __syncwarp();
      if (lane == 0) {
        if constexpr (MB)
          for (int x = xb; x < xe; x++) mbar_arrive(&full_bar[kWRows * kWRing + (x & (kWRing - 1))]);
        else
          st_release_cta(&prog[kWRows], xe);
      }
    }
    return;
  }
  if (w == kWRows + 1) {
    // ---------------- publisher: the block's last row into the global band buffer ----------------
    if (below_exists) {
      int seen = 0;
      for (int x = 0; x < W; x++) {
        if (MB ? !wait_full(kWRows - 1, x) : !wait(kWRows - 1, x + 1, seen)) break;
        const int sl = x & (kWRing - 1);
#pragma unroll
        for (int p = 0; p < 3; p++) {
          V<LPT> v;
          sload<LPT>(v, vec(kWRows - 1, sl, p), lane);
          vstore<LPT>(v, bnd_me + ((size_t)x * 3 + p) * Dp, lane);
        }
        if (lane == 0) __stcg(bnd_me_md + x, mrec(kWRows - 1, sl));
        __syncwarp();
        if (lane == 0) {
          st_release_cta(&prog[kWRows + 1], x + 1);                                   // the slot is free again
          if ((x + 1) % kWPublish == 0) st_release(a.progress + cb, x + 1);           // the next block's loader polls this
        }
      }
    }
    __syncwarp();
    if (lane == 0) st_release(a.progress + cb, W);
    return;
  }

  // ---------------- a row of the recurrence ----------------
  if (w >= rows) return;
  const int y = y0 + w;  // row of the pass
  const int up = w == 0 ? kWRows : w - 1;                             // the set holding the row above
  const int cons_idx = w + 1 < kWRows ? w + 1 : kWRows + 1;          // who reads this row's set
  const bool has_consumer = y + 1 < a.H;
  const uint32_t p1x2 = dup16((uint32_t)a.p1);
  const int yu = PASS2 ? a.H - 1 - y : y;
  const uint8_t* raw_row = a.raw + (size_t)yu * W * a.n + lane * LPT;
  uint16_t* agg_row = a.agg + (size_t)yu * W * a.n + lane * LPT;
  const uint2* p2_row = a.p2t + (size_t)y * W;
  float* depth_row = a.depth + (size_t)yu * W;
  const int flags = a.flags[y];
  const bool edge_row = !PASS2 && y == a.y_b;  // pass +1's row y_b is what pass -1 reads above its first row
  int seen_up = MB ? -1 : 0, seen_cons = 0;
  V<LPT> leftL;   // path 0: the pixel to the left
  uint32_t leftm = kInit2;
  vinit(leftL);
  struct Queued {  // what a pixel reads from HBM, fetched two pixels ahead
    RawB<LPT> raw;
    V<LPT> agg;  // pass -1: pass +1's aggregates
    uint2 p2;
  };
  auto col_of = [&](int x) { return PASS2 ? c - x : x; };
  auto fetch = [&](int xq, Queued& q) {
    const int off = col_of(xq) * a.n;
    const uint8_t* rp = raw_row + off;
    if (!active) {
      q.raw.r[0] = 0;
      if constexpr (LPT >= 8) q.raw.r[1] = 0;
    } else if constexpr (LPT == 8) {
      const uint2 t = __ldcs(reinterpret_cast<const uint2*>(rp));
      q.raw.r[0] = t.x;
      q.raw.r[1] = t.y;
    } else if constexpr (LPT == 4) {
      q.raw.r[0] = __ldcs(reinterpret_cast<const unsigned int*>(rp));
    } else {
      q.raw.r[0] = __ldcs(reinterpret_cast<const unsigned short*>(rp));
    }
    if constexpr (PASS2) agg_load<LPT>(agg_row + off, q.agg, active);
    q.p2 = __ldg(p2_row + xq);
  };
  // One visit N(x, y). KIND: 0 the first column, 1 a column with both neighbours and no revisit business, 2 the column
  // c-1 (its path states 0 and 1 are kept for the revisits), 3 the last column c (revisits, the special path-2 read).
  auto pixel = [&](int x, Queued& q, auto kind) -> bool {
    constexpr int KIND = decltype(kind)::value;
    // ---- hand-over in: the row above finished x+1 (x for the last column); the next row is done with this slot ----
    if constexpr (MB) {
      const int tp = min(x + 1, c);  // the row above's pixel x+1 (the last column: its own)
      if (tp > seen_up) {
        if (!wait_full(up, tp)) return false;
        seen_up = tp;
      }
    } else {
      if (!wait(up, min(x + 2, W), seen_up)) return false;
    }
    if (has_consumer && x >= kWRing && !wait(cons_idx, x - kWRing + 2 - (cons_idx == kWRows + 1 ? 1 : 0), seen_cons))
      return false;
    // ---- revisits that the reference runs before this visit (they may produce this visit's path-2 input) ----
    if constexpr (KIND == 3) {
      const int cnt = a.batch_count[y], first = a.batch_first[y];
      for (int k = 0; k < cnt; k++) run_revisit<LPT>(a, first + k, lane, active);
    }
    // ---- neighbour states: path 0 the pixel to the left, paths 1, 2, 3 pixels x-1, x, x+1 of row y-1 ----
    V<LPT> nb[4];
    uint32_t md[4];
    nb[0] = leftL;
    md[0] = leftm;
#pragma unroll
    for (int p = 1; p < 4; p++) {
      if ((KIND == 0 && p == 1) || (KIND == 3 && p == 3)) {  // outside the image: a never-written slot
        vinit(nb[p]);
        md[p] = kInit2;
        continue;
      }
      const int sl = (x + p - 2) & (kWRing - 1);
      sload<LPT>(nb[p], vec(up, sl, p - 1), lane);
      const uint4& mr = mrec(up, sl);
      md[p] = p == 1 ? mr.x : p == 2 ? mr.y : mr.z;
    }
    if constexpr (KIND == 3) {
      if (flags & 1) {  // N(c).p2 reads R(c, y-1)
        Src<LPT> r;
        src_cs<LPT>(a, r, y - 1, 4, c, lane);
        nb[2] = r.L;
        md[2] = dup16(r.mn);
      }
    }
    // ---- the four paths ----
    V<LPT> raw2, acc, out[4];
    raw_unpack<LPT>(q.raw, raw2);
    if constexpr (PASS2) {
      acc = q.agg;
    } else {
#pragma unroll
      for (int i = 0; i < NR; i++) acc.r[i] = 0;
    }
    uint32_t mdo[4];
    wave_paths<LPT, FULL>(nb, md, q.p2, p1x2, raw2, active, lane, out, acc, mdo);
    // ---- hand-over out: the ring slot, then the release; global stores after it ----
    const int sl = x & (kWRing - 1);
#pragma unroll
    for (int p = 1; p < 4; p++) sstore<LPT>(out[p], vec(w, sl, p - 1), lane);
    if (lane == 0) mrec(w, sl) = make_uint4(mdo[1], mdo[2], mdo[3], 0u);
    uint16_t* ap = agg_row + col_of(x) * a.n;
    if constexpr (KIND == 2) {  // what later revisits read is stored before the release
      cs_put<LPT>(a, out[0], mdo[0] & 0xffffu, y, 0, lane);
      cs_put<LPT>(a, out[1], mdo[1] & 0xffffu, y, 1, lane);
    }
    if constexpr (KIND == 3) {
      cs_put<LPT>(a, out[2], mdo[2] & 0xffffu, y, 2, lane);
      agg_store<LPT>(ap, acc, active);
    }
    __syncwarp();
    if (lane == 0) {
      if constexpr (MB) mbar_arrive(&full_bar[w * kWRing + sl]);
      st_release_cta(&prog[w], x + 1);
    }
    if constexpr (KIND != 3) {
      if (!PASS2 || a.keep_agg) agg_store<LPT>(ap, acc, active);
      if constexpr (PASS2) {  // WTA; the last column waits for its revisits (k_wta_column)
        const int arg = wta_arg<LPT>(acc, active, lane);
        if (lane == 0) depth_row[col_of(x)] = s_planes[arg];
      }
    }
    if (edge_row) {
#pragma unroll
      for (int p = 1; p < 4; p++) {
        vstore<LPT>(out[p], a.edge + ((size_t)x * 3 + (p - 1)) * Dp, lane);
        if (lane == 0) __stcg(a.edge_min + (size_t)x * 3 + (p - 1), (uint16_t)(mdo[p] & 0xffffu));
      }
    }
    if constexpr (KIND == 3) {
      if (y == a.H - 1)  // the last band's revisits when no later visit of the column follows them
        for (int k = 0; k < a.end_count; k++) run_revisit<LPT>(a, a.end_first + k, lane, active);
    }
    leftL = out[0];
    leftm = mdo[0];
    if constexpr (KIND <= 1) fetch(x + 2, q);  // x + 2 <= c
    return true;
  };
  using K0 = std::integral_constant<int, 0>;
  using K1 = std::integral_constant<int, 1>;
  using K2 = std::integral_constant<int, 2>;
  using K3 = std::integral_constant<int, 3>;
  // Pixel x reads queue entry x & 1, so the two-deep prefetch needs no register moves.
  Queued q0, q1;
  fetch(0, q0);
  fetch(1, q1);
  if (!pixel(0, q0, K0{})) return;
  int x = 1;
  for (; x + 1 <= c - 2; x += 2) {
    if (!pixel(x, q1, K1{})) return;
    if (!pixel(x + 1, q0, K1{})) return;
  }
  if (x <= c - 2) {
    if (!pixel(x, q1, K1{})) return;
    x++;
  }
  if (x & 1) {
    if (pixel(c - 1, q1, K2{})) pixel(c, q0, K3{});
  } else {
    if (pixel(c - 1, q0, K2{})) pixel(c, q1, K3{});
  }
}

struct WaveLayout {
  size_t bnd, bnd_md, progress, edge, edge_min, cs, cs_min, sched, p2t, total;
};

WaveLayout wave_layout(int W, int H, int n) {
  const size_t Dp = 32 * (size_t)(n <= 64 ? 2 : n <= 128 ? 4 : 8);
  const int nCB = (H + kWRows - 1) / kWRows;
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  WaveLayout L;
  size_t o = 0;
  L.bnd = o; o += al((size_t)kWBandBufs * W * 3 * Dp * 2);
  L.bnd_md = o; o += al((size_t)kWBandBufs * W * 16);
  L.progress = o; o += al((size_t)(nCB + 2) * 4 * 2);
  L.edge = o; o += al((size_t)W * 3 * Dp * 2);
  L.edge_min = o; o += al((size_t)W * 3 * 2);
  L.cs = o; o += al((size_t)H * 5 * Dp * 2);
  L.cs_min = o; o += al((size_t)H * 5 * 2);
  L.sched = o; o += al((size_t)2 * 7 * H * 4);
  L.p2t = o; o += al((size_t)W * H * 8);
  L.total = o;
  return L;
}

template <int LPT, bool FULL, bool PASS2, bool MB>
void launch_wave_tm(const WaveArgs& wa, int nCB, cudaStream_t s) {
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_wave<LPT, FULL, PASS2, MB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wave_smem_bytes<LPT>());
    configured = true;
  }
  k_wave<LPT, FULL, PASS2, MB><<<nCB, kWWarps * 32, wave_smem_bytes<LPT>(), s>>>(wa);
  count_launches(1);
}
// The hand-over in waits on the ring slots' full mbarriers (MB = true): measured faster than polling the row counters
// (MB = false, which the kernel keeps as the plain form of the same schedule).
template <int LPT, bool FULL, bool PASS2>
void launch_wave_t(const WaveArgs& wa, int nCB, cudaStream_t s) {
  launch_wave_tm<LPT, FULL, PASS2, true>(wa, nCB, s);
}
template <int LPT>
void launch_wave(const WaveArgs& wa, int nCB, cudaStream_t s) {
  const bool full = wa.u.n == 32 * LPT;
  if (wa.u.dir > 0) {
    if (full) launch_wave_t<LPT, true, false>(wa, nCB, s);
    else launch_wave_t<LPT, false, false>(wa, nCB, s);
  } else {
    if (full) launch_wave_t<LPT, true, true>(wa, nCB, s);
    else launch_wave_t<LPT, false, true>(wa, nCB, s);
  }
}

}  // namespace

// k_p2_table and k_wta_column live in sgm_uniform.cu
void launch_p2_table(const UniArgs& a, uint2* p2t, cudaStream_t s);
void launch_wta_column(const uint16_t* agg, int W, int H, int n, const float* planes, float* depth, cudaStream_t s);

size_t wave_scratch_bytes(int W, int H, int n) { return wave_layout(W, H, n).total; }

int run_sgm_wave(const LayerGeom& g, int xsw, uint16_t p1, float p2scale, const float gw[4], const uint8_t* raw, uint16_t* agg,
                 uint16_t* agg_pass1, float* depth, int keep_agg, void* scratch, size_t scratch_bytes, int* err, cudaStream_t s) {
  if (xsw) return 12;  // LUX_SGM_XSW changes the traversal; the replay kernel covers it
  const int W = g.W, H = g.H, n = g.n_planes, T = g.tile;
  const WaveLayout L = wave_layout(W, H, n);
  if (scratch_bytes < L.total) return 9;
  char* base = static_cast<char*>(scratch);
  RevisitSchedule sch[2];
  std::vector<int> host((size_t)2 * 7 * H);
  for (int pass = 0; pass < 2; pass++) {
    build_revisit_schedule(W, H, T, pass == 1, sch[pass]);
    int* h = host.data() + (size_t)pass * 7 * H;
    const std::vector<int>* cols[7] = {&sch[pass].flags, &sch[pass].batch_first, &sch[pass].batch_count, &sch[pass].src0,
                                       &sch[pass].src1, &sch[pass].src2, &sch[pass].extra};
    for (int k = 0; k < 7; k++) std::memcpy(h + (size_t)k * H, cols[k]->data(), (size_t)H * 4);
  }
  int* dsched = reinterpret_cast<int*>(base + L.sched);
  if (cudaMemcpyAsync(dsched, host.data(), host.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return 10;
  const int nCB = (H + kWRows - 1) / kWRows;
  int* progress = reinterpret_cast<int*>(base + L.progress);
  cudaMemsetAsync(progress, 0, (size_t)(nCB + 2) * 4 * 2, s);
  WaveArgs wa;
  std::memset(&wa, 0, sizeof wa);
  UniArgs& a = wa.u;
  a.W = W; a.H = H; a.n = n; a.T = T; a.nCB = nCB;
  a.raw = raw; a.agg = agg; a.depth = depth; a.planes = g.planes; a.guidance = g.guidance;
  a.p1 = p1;
  volatile float p1f = (float)p1;
  a.p2base = p1f * p2scale;
  for (int i = 0; i < 4; i++) a.gw[i] = gw[i];
  wa.bnd = reinterpret_cast<uint16_t*>(base + L.bnd);
  wa.bnd_md = reinterpret_cast<uint4*>(base + L.bnd_md);
  a.edge = reinterpret_cast<uint16_t*>(base + L.edge);
  a.edge_min = reinterpret_cast<uint16_t*>(base + L.edge_min);
  a.cs = reinterpret_cast<uint16_t*>(base + L.cs);
  a.cs_min = reinterpret_cast<uint16_t*>(base + L.cs_min);
  a.y_b = sch[0].y_b;
  a.err = err;
  a.timeout_ns = g.timeout_ns;
  a.stall_block = g.stall_block;
  a.never = g.never;
  a.keep_agg = keep_agg;
  a.p2t = reinterpret_cast<const uint2*>(base + L.p2t);
  const int lpt = n <= 64 ? 2 : n <= 128 ? 4 : 8;
  for (int pass = 0; pass < 2; pass++) {
    const int* h = dsched + (size_t)pass * 7 * H;
    a.flags = h; a.batch_first = h + H; a.batch_count = h + 2 * H; a.src0 = h + 3 * H; a.src1 = h + 4 * H; a.src2 = h + 5 * H;
    a.extra = h + 6 * H;
    a.end_first = sch[pass].end_first;
    a.end_count = sch[pass].end_count;
    a.dir = pass == 0 ? 1 : -1;
    a.progress = progress + (size_t)pass * (nCB + 2);
    a.ticket = progress + (size_t)pass * (nCB + 2) + nCB;
    a.edge_write = pass == 0;
    a.edge_read = pass == 1;
    a.wta = pass == 1;
    launch_p2_table(a, reinterpret_cast<uint2*>(base + L.p2t), s);
    if (lpt == 2) launch_wave<2>(wa, nCB, s);
    else if (lpt == 4) launch_wave<4>(wa, nCB, s);
    else launch_wave<8>(wa, nCB, s);
    if (pass == 0 && agg_pass1) cudaMemcpyAsync(agg_pass1, agg, (size_t)W * H * n * 2, cudaMemcpyDeviceToDevice, s);
  }
  launch_wta_column(agg, W, H, n, g.planes, depth, s);
  return 0;
}

}  // namespace lux
