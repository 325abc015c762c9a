// Fast aggregation of a uniform layer (every pixel searches planes [0, n), the first layer of a pyramid and every
// plain pair): bit-exact with the reference's traversal (DenseStereoSgm.cs:181-324) through revisit_schedule.h.
//
// Shape: a CTA owns kRows consecutive rows of a pass (mirrored coordinates in pass -1), one warp per row. Row y handles
// pixel x once row y-1 has finished x+1, so the rows of a block run as a wavefront two pixels apart. All four paths of
// a pixel are fused, so each pass reads the raw volume once and touches the aggregates once:
//   pass +1: agg = sum of paths;  pass -1: agg += sum of paths, then WTA (the aggregates are stored only when kept).
// A lane owns LPT consecutive planes as LPT/2 packed u16 pairs: min.u16x2 for the four-way minimum, byte permutes for
// the d±1 neighbours, one shuffle per side across lanes, and redux.sync for the running minimum.
// Hand-over: each row writes its path states 1-3 into a kRing-slot shared-memory ring; the row below waits on the
// slot's full mbarrier and frees it through its empty mbarrier (waiting warps are suspended by the hardware, not
// spinning). A loader warp fills the ring of the row above the block from a global band buffer, gated by the previous
// block's progress counter; a publisher warp copies the block's last row out and releases its own counter every
// kPublish pixels. Blocks take tickets in order, so a block only ever waits on a block that is already running; every
// wait is bounded and a timeout stops the block with error 11.
//
// Exactness without saturation: with P2 <= p2base <= 1744 every stored L is at most 255 + 1744 < 2000 (the value of a
// never-written word), the running minimum is at most 2000, and every candidate of the four-way minimum is at least
// the previous minimum, so raw + m - minPrev never leaves [0, 65535] and 16 path contributions never exceed 65535.
#include <cstring>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "revisit_schedule.h"
#include "sgm_paths.cuh"

namespace lux {

// kRows: rows of the recurrence per block (one warp each), kWarps: plus the loader and the publisher warps, kRing: slots
// of the hand-over ring between neighbouring rows of a block. Past 256 planes (LPT 16 or 24) a ring slot holds 32·LPT
// planes of three paths, so the block runs 4 rows to keep its rings in an SM's shared memory (184 KB at LPT 24). The
// ring keeps 8 slots: the loader frees a batch of 4 slots before it fills them, which a ring of 4 could never do while
// row 0 holds the slots of the pixels it reads.
template <int LPT>
struct UniCfg {
  static constexpr int kRows = LPT > 8 ? 4 : 14;
  static constexpr int kRing = 8;
  static constexpr int kWarps = kRows + 2;
};
constexpr int uni_rows(int lpt) { return lpt > 8 ? UniCfg<16>::kRows : UniCfg<8>::kRows; }
constexpr int kBandBufs = 4;   // band buffers in rotation
constexpr int kPublish = 8;    // the publisher releases the global band progress every kPublish pixels

// Shared memory of a block: kRows + 1 hand-over rings (ring kRows is the row above the block, filled by the loader warp),
// their minima, and a full and an empty mbarrier per ring slot.
template <int LPT>
constexpr size_t ring_bytes() {
  constexpr int kRows = UniCfg<LPT>::kRows, kRing = UniCfg<LPT>::kRing;
  return (size_t)(kRows + 1) * kRing * 3 * Dp_of(LPT) * 2 + (size_t)(kRows + 1) * kRing * 3 * 2 + 16 +
         (size_t)2 * (kRows + 1) * kRing * 8;
}

// Guidance of the path-p neighbour of pixel (xq, yq) of the pass: margins and never-written slots give 0; the row above
// the first row is pass +1's row y_b in pass -1 (its final line buffer) and never written in pass +1.
LUX_DEV float4 neighbour_pix(const UniArgs& a, int p, int xq, int yq) {
  const int xn = xq + (p == 0 || p == 1 ? -1 : p == 2 ? 0 : 1);
  const int yn = p == 0 ? yq : yq - 1;
  if (xn < 0 || xn >= a.W) return make_float4(0.f, 0.f, 0.f, 0.f);
  if (yn < 0) {
    if (!a.edge_read || a.y_b < 0) return make_float4(0.f, 0.f, 0.f, 0.f);
    return pix_edge(a, a.dir > 0 ? xn : a.W - 1 - xn);
  }
  return pix_of(a, xn, yn);
}

// The four P2 values of every pixel of a pass (DenseStereoSgm.cs:266-273): they depend only on the guidance image (and
// at the first row of pass -1 on pass +1's row y_b), so they are computed once per pass, packed as u16 (P2 <= 1744).
__global__ void k_p2_table(const UniArgs a, uint2* __restrict__ p2t) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= a.W) return;
  const float4 g = pix_of(a, x, y);
  uint32_t v[4];
#pragma unroll
  for (int p = 0; p < 4; p++) v[p] = (uint32_t)p2_of(a, g, neighbour_pix(a, p, x, y));
  p2t[(size_t)y * a.W + x] = make_uint2(v[0] | (v[1] << 16), v[2] | (v[3] << 16));
}

// The row above a block, pixel by pixel, as the block's first row reads it: the last row of the block above (from the
// global band buffer), pass +1's final line buffer at the first row of pass -1, or never-written slots.
template <int LPT>
LUX_DEV void row_above(const UniArgs& a, const uint16_t* bnd_up, const uint16_t* bnd_up_min, int cb, int x, Src<LPT> (&u)[3], int lane) {
  constexpr int Dp = Dp_of(LPT);
#pragma unroll
  for (int p = 1; p < 4; p++) {
    if (cb > 0) {
      vload<LPT>(u[p - 1].L, bnd_up + ((size_t)x * 3 + (p - 1)) * Dp, lane);
      u[p - 1].mn = __ldcg(bnd_up_min + (size_t)x * 3 + (p - 1));
    } else if (a.edge_read) {
      src_edge<LPT>(a, u[p - 1], a.dir > 0 ? x : a.W - 1 - x, p, lane);
    } else {
      src_init(u[p - 1]);
    }
  }
}

// Warps 0..kRows-1 run the recurrence of one row each; warp kRows (loader) brings the row above the block into ring
// kRows; warp kRows+1 (publisher) copies the block's last row to the global band buffer for the block below. A row
// waits only on its neighbours (shared-memory acquire/release), so the global latencies of the block boundary stay
// off the rows' own critical path.
template <int LPT, bool FULL, bool PASS2>
__global__ void __launch_bounds__(UniCfg<LPT>::kWarps * 32, 1) k_sgm_uniform(const UniArgs a) {
  constexpr int NR = LPT / 2, Dp = Dp_of(LPT), kBatch = 4;
  constexpr int kRows = UniCfg<LPT>::kRows, kRing = UniCfg<LPT>::kRing, kWarps = UniCfg<LPT>::kWarps;
  static_assert(kBatch < kRing, "the loader frees a batch of slots before filling them");
  extern __shared__ __align__(16) uint16_t smem_ring[];
  auto ring = [&](int set, int slot, int p) { return smem_ring + (((size_t)set * kRing + slot) * 3 + p) * Dp; };
  uint16_t* ring_min = smem_ring + (size_t)(kRows + 1) * kRing * 3 * Dp;
  auto rmin_at = [&](int set, int slot, int p) -> uint16_t& { return ring_min[((size_t)set * kRing + slot) * 3 + p]; };
  // full(set, slot): the producer of ring `set` filled the slot; empty(set, slot): its consumer is done with it
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring_min + (size_t)(kRows + 1) * kRing * 3 + 8);
  auto full = [&](int set, int slot) { return bars + set * kRing + slot; };
  auto empty = [&](int set, int slot) { return bars + (kRows + 1) * kRing + set * kRing + slot; };
  __shared__ int s_cb;
  __shared__ volatile int s_stop;
  __shared__ float s_planes[LPT > 8 ? 32 * LPT : 256];  // the WTA's plane depths (pass -1)
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (PASS2)
    for (int i = tid; i < a.n; i += blockDim.x) s_planes[i] = a.planes[i];
  if (tid == 0) {
    s_cb = atomicAdd(a.ticket, 1);
    s_stop = 0;
  }
  static_assert(kWarps * 32 >= 2 * (kRows + 1) * kRing, "one thread per mbarrier");
  if (tid < 2 * (kRows + 1) * kRing) mbar_init(bars + tid, 1);
  __syncthreads();
  const int cb = s_cb;
  const int y0 = cb * kRows;
  const bool below_exists = y0 + kRows < a.H;  // a block below reads this block's last row
  const int active = FULL ? (LPT > 8 ? LPT / 8 : 1) : lane_octets<LPT>(a.n, lane);  // planes in use, in octets
  const uint16_t* bnd_up = a.bnd + (size_t)((cb + kBandBufs - 1) % kBandBufs) * a.W * 3 * Dp;
  const uint16_t* bnd_up_min = a.bnd_min + (size_t)((cb + kBandBufs - 1) % kBandBufs) * a.W * 3;
  uint16_t* bnd_me = a.bnd + (size_t)(cb % kBandBufs) * a.W * 3 * Dp;
  uint16_t* bnd_me_min = a.bnd_min + (size_t)(cb % kBandBufs) * a.W * 3;
  // Slot x & (kRing - 1) of a ring holds pixel x; it completes phase x / kRing of its full barrier when filled and,
  // once the consumer is done with it, phase x / kRing of its empty barrier. Waits are bounded: a timeout stops the
  // block (error 11) and every other wait of the block then gives up.
  auto wait_filled = [&](int set, int x) {  // pixel x of ring `set` is there
    return mbar_wait(full(set, x & (kRing - 1)), (uint32_t)(x / kRing) & 1u, &s_stop, a.err, a.timeout_ns);
  };
  auto wait_free = [&](int set, int x) {  // the slot of pixel x no longer holds pixel x - kRing for the consumer
    return x < kRing || mbar_wait(empty(set, x & (kRing - 1)), (uint32_t)(x / kRing - 1) & 1u, &s_stop, a.err, a.timeout_ns);
  };

  if (w == kRows) {
    // ---------------- loader: the row above the block into ring kRows ----------------
    if (y0 < a.H) {
      // pixels of the block above known to be published: the counter is polled only when the loader has caught up with
      // it, and then up to kBatch pixels are loaded at once, so their L2 round trips overlap
      int avail = cb > 0 ? 0 : a.W;
      for (int xb = 0; xb < a.W && !s_stop; xb += kBatch) {
        const int xe = min(a.W, xb + kBatch);
        bool ok = true;
        for (int x = xb; x < xe && ok; x++) ok = wait_free(kRows, x);  // row 0 is done with these slots
        if (!ok) break;
        if (avail < xe) {
          int v = 0;
          if (lane == 0) v = wait_at_least_value(cb == a.stall_block ? a.never : a.progress + (cb - 1), xe, a.err, 11, a.timeout_ns);
          v = __shfl_sync(0xffffffffu, v, 0);
          __syncwarp();  // lane 0's acquire orders the band-buffer reads of every lane
          if (v < 0) {
            s_stop = 1;
            break;
          }
          avail = v;
        }
        Src<LPT> u[kBatch][3];
#pragma unroll
        for (int k = 0; k < kBatch; k++)
          if (xb + k < xe) row_above<LPT>(a, bnd_up, bnd_up_min, cb, xb + k, u[k], lane);
#pragma unroll
        for (int k = 0; k < kBatch; k++) {
          if (xb + k >= xe) break;
          const int sl = (xb + k) & (kRing - 1);
#pragma unroll
          for (int p = 0; p < 3; p++) {
            vstore_s<LPT>(u[k][p].L, ring(kRows, sl, p), lane);
            if (lane == 0) rmin_at(kRows, sl, p) = (uint16_t)u[k][p].mn;
          }
        }
        __syncwarp();
        if (lane == 0)
          for (int x = xb; x < xe; x++) mbar_arrive(full(kRows, x & (kRing - 1)));
      }
    }
    return;
  }
  if (w == kRows + 1) {
    // ---------------- publisher: the block's last row into the global band buffer ----------------
    if (below_exists) {
      for (int x = 0; x < a.W; x++) {
        if (!wait_filled(kRows - 1, x)) break;
        const int sl = x & (kRing - 1);
#pragma unroll
        for (int p = 0; p < 3; p++) {
          V<LPT> v;
          vload_s<LPT>(v, ring(kRows - 1, sl, p), lane);
          vstore<LPT>(v, bnd_me + ((size_t)x * 3 + p) * Dp, lane);
          if (lane == 0) __stcg(bnd_me_min + (size_t)x * 3 + p, rmin_at(kRows - 1, sl, p));
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(empty(kRows - 1, x & (kRing - 1)));  // the ring slot is free again
        if ((x + 1) % kPublish == 0) st_release(a.progress + cb, x + 1);  // the next block's loader polls this
      }
    }
    __syncwarp();
    if (lane == 0) st_release(a.progress + cb, a.W);
    return;
  }

  // ---------------- a row of the recurrence ----------------
  const int y = y0 + w;  // row of the pass
  if (y >= a.H) return;
  const int up_set = w == 0 ? kRows : w - 1;  // the ring holding the row above
  const bool has_consumer = y + 1 < a.H;
  const int c = a.W - 1;
  const uint32_t p1x2 = dup16((uint32_t)a.p1);
  const int yu = PASS2 ? a.H - 1 - y : y;
  const uint8_t* raw_row = a.raw + (size_t)yu * a.W * a.n + lane * LPT;
  uint16_t* agg_row = a.agg + (size_t)yu * a.W * a.n + lane * LPT;
  const uint2* p2_row = a.p2t + (size_t)y * a.W;
  float* depth_row = a.depth + (size_t)yu * a.W;
  const int flags = a.flags[y];
  const bool edge_row = !PASS2 && y == a.y_b;  // pass +1's row y_b is what pass -1 reads above its first row
  Src<LPT> left;  // path 0: the pixel to the left
  src_init(left);
  struct Queued {  // what a pixel reads from HBM, fetched two pixels ahead
    RawB<LPT> raw;
    V<LPT> agg;  // pass -1: pass +1's aggregates
    uint2 p2;
  };
  // pixel x of the pass is image column col_of(x); 32-bit offsets (W·n < 2^31) keep the addressing to a few adds
  auto col_of = [&](int x) { return PASS2 ? c - x : x; };
  auto fetch = [&](int xq, Queued& q) {
    const int off = col_of(xq) * a.n;
    const uint8_t* rp = raw_row + off;
    if constexpr (LPT > 8) {  // the octets in use, 8 bytes each
#pragma unroll
      for (int o = 0; o < LPT / 8; o++) {
        const uint2 t = o < active ? __ldcs(reinterpret_cast<const uint2*>(rp) + o) : make_uint2(0u, 0u);
        q.raw.r[2 * o] = t.x;
        q.raw.r[2 * o + 1] = t.y;
      }
    } else if (!active) {
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
    // ---- hand-over in: the row above finished x+1; the next row is done with the ring slot this pixel reuses ----
    if constexpr (KIND != 3) {
      if (!wait_filled(up_set, x + 1)) return false;
    }
    if (has_consumer && !wait_free(w, x)) return false;
    // ---- revisits that the reference runs before this visit (they may produce this visit's path-2 input) ----
    if constexpr (KIND == 3) {
      const int cnt = a.batch_count[y], first = a.batch_first[y];
      for (int k = 0; k < cnt; k++) run_revisit<LPT>(a, first + k, lane, active);
    }
    // ---- neighbour states: path 0 the pixel to the left, paths 1, 2, 3 pixels x-1, x, x+1 of row y-1 ----
    V<LPT> nbL[4];
    uint32_t mp[4];
    nbL[0] = left.L;
    mp[0] = left.mn;
#pragma unroll
    for (int p = 1; p < 4; p++) {
      if ((KIND == 0 && p == 1) || (KIND == 3 && p == 3)) {  // outside the image: a never-written slot
        vinit(nbL[p]);
        mp[p] = 2000;
        continue;
      }
      const int sl = (x + p - 2) & (kRing - 1);
      vload_s<LPT>(nbL[p], ring(up_set, sl, p - 1), lane);
      mp[p] = rmin_at(up_set, sl, p - 1);
    }
    if constexpr (KIND == 3) {
      if (flags & 1) {  // N(c).p2 reads R(c, y-1)
        Src<LPT> r;
        src_cs<LPT>(a, r, y - 1, 4, c, lane);
        nbL[2] = r.L;
        mp[2] = r.mn;
      }
    }
    // ---- the four paths ----
    const uint32_t p2[4] = {q.p2.x & 0xffffu, q.p2.x >> 16, q.p2.y & 0xffffu, q.p2.y >> 16};
    V<LPT> raw2, acc, out[4];
    raw_unpack<LPT>(q.raw, raw2);
    if constexpr (PASS2) {
      acc = q.agg;
    } else {
#pragma unroll
      for (int i = 0; i < NR; i++) acc.r[i] = 0;
    }
    uint32_t mins[4];
    four_paths<LPT, FULL>(nbL, mp, p2, p1x2, raw2, active, lane, out, acc, mins);
    // ---- hand-over out: the ring first, then the release; global stores after it ----
    const int sl = x & (kRing - 1);
#pragma unroll
    for (int p = 1; p < 4; p++) {
      vstore_s<LPT>(out[p], ring(w, sl, p - 1), lane);
      if (lane == 0) rmin_at(w, sl, p - 1) = (uint16_t)mins[p];
    }
    uint16_t* ap = agg_row + col_of(x) * a.n;
    if constexpr (KIND == 2) {  // what later revisits of this block read is stored before the release
      cs_put<LPT>(a, out[0], mins[0], y, 0, lane);
      cs_put<LPT>(a, out[1], mins[1], y, 1, lane);
    }
    if constexpr (KIND == 3) {
      cs_put<LPT>(a, out[2], mins[2], y, 2, lane);
      agg_store<LPT>(ap, acc, active);
    }
    __syncwarp();
    if (lane == 0) {
      mbar_arrive(full(w, sl));                                                          // pixel x is in the ring
      if constexpr (KIND != 0) mbar_arrive(empty(up_set, (x - 1) & (kRing - 1)));  // the row above's x-1 is done
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
        if (lane == 0) __stcg(a.edge_min + (size_t)x * 3 + (p - 1), (uint16_t)mins[p]);
      }
    }
    if constexpr (KIND == 3) {
      if (y == a.H - 1)  // the last band's revisits when no later visit of the column follows them
        for (int k = 0; k < a.end_count; k++) run_revisit<LPT>(a, a.end_first + k, lane, active);
    }
    left.L = out[0];
    left.mn = mins[0];
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

// WTA of the last column of pass -1 (its aggregates are final only after the revisits).
__global__ void k_wta_column(const uint16_t* __restrict__ agg, int W, int H, int n, int col, const float* __restrict__ planes,
                             float* __restrict__ depth) {
  const int y = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (y >= H) return;
  const uint16_t* p = agg + ((size_t)y * W + col) * n;
  int best = 0xffff, arg = 0x7fffffff;
  for (int k = lane; k < n; k += 32) {
    int v = p[k];
    if (v < best) { best = v; arg = k; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    int ob = __shfl_xor_sync(0xffffffffu, best, o), oa = __shfl_xor_sync(0xffffffffu, arg, o);
    if (ob < best || (ob == best && oa < arg)) { best = ob; arg = oa; }
  }
  if (lane == 0) depth[(size_t)y * W + col] = planes[arg == 0x7fffffff ? 0 : arg];
}

void launch_p2_table(const UniArgs& a, uint2* p2t, cudaStream_t s) {
  k_p2_table<<<dim3((a.W + 127) / 128, a.H), 128, 0, s>>>(a, p2t);
  count_launches(1);
}
void launch_wta_column(const uint16_t* agg, int W, int H, int n, const float* planes, float* depth, cudaStream_t s) {
  k_wta_column<<<(H * 32 + 255) / 256, 256, 0, s>>>(agg, W, H, n, 0, planes, depth);
  count_launches(1);
}

size_t uniform_supported_planes() { return 256; }  // the chain and wave forms; the fused form takes up to 768
bool uniform_wide_planes(int n) { return n > 256; }

static int lpt_for(int n) { return n <= 64 ? 2 : n <= 128 ? 4 : n <= 256 ? 8 : n <= 512 ? 16 : 24; }

bool uniform_fast_supported(int W, int H, int n, int tile, uint16_t p1, float p2scale) {
  if (n <= 0 || n > 768 || (n & 7) != 0) return false;  // past 256 planes the fused form only (uniform_wide_planes)
  if ((tile & 1) != 0 || tile < 2) return false;  // a row's half of the line buffer is its parity only for even tiles
  if (W < 3 || H < 2) return false;
  volatile float p1f = (float)p1;
  const float p2base = p1f * p2scale;
  if (!(p2scale >= 0.0f) || !(p2base <= 1744.0f) || p1 > 60000) return false;  // the no-saturation bound above
  return true;
}

struct UniScratchLayout {
  size_t bnd, bnd_min, progress, edge, edge_min, cs, cs_min, sched, p2t, total;
};

static UniScratchLayout layout_of(int W, int H, int n) {
  const size_t Dp = 32 * (size_t)lpt_for(n);
  const int rows = uni_rows(lpt_for(n));
  const int nCB = (H + rows - 1) / rows;
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  UniScratchLayout L;
  size_t o = 0;
  L.bnd = o; o += al((size_t)kBandBufs * W * 3 * Dp * 2);
  L.bnd_min = o; o += al((size_t)kBandBufs * W * 3 * 2);
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

size_t uniform_scratch_bytes(int W, int H, int n, int tile) {
  (void)tile;
  return layout_of(W, H, n).total;
}

template <int LPT, bool FULL, bool PASS2>
static void launch_pass_t(const UniArgs& a, cudaStream_t s) {
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_sgm_uniform<LPT, FULL, PASS2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ring_bytes<LPT>());
    configured = true;
  }
  k_sgm_uniform<LPT, FULL, PASS2><<<a.nCB, UniCfg<LPT>::kWarps * 32, ring_bytes<LPT>(), s>>>(a);
  count_launches(1);
}
template <int LPT>
static void launch_pass(const UniArgs& a, cudaStream_t s) {
  const bool full = a.n == 32 * LPT;
  if (a.dir > 0) {
    if (full) launch_pass_t<LPT, true, false>(a, s);
    else launch_pass_t<LPT, false, false>(a, s);
  } else {
    if (full) launch_pass_t<LPT, true, true>(a, s);
    else launch_pass_t<LPT, false, true>(a, s);
  }
}

int run_sgm_uniform(const LayerGeom& g, int xsw, uint16_t p1, float p2scale, const float gw[4], const uint8_t* raw, uint16_t* agg,
                    uint16_t* agg_pass1, float* depth, int keep_agg, void* scratch, size_t scratch_bytes, int* err,
                    cudaStream_t s) {
  if (xsw) return 12;  // LUX_SGM_XSW changes the traversal; the replay kernel covers it
  const int W = g.W, H = g.H, n = g.n_planes, T = g.tile;
  const UniScratchLayout L = layout_of(W, H, n);
  if (scratch_bytes < L.total) return 9;
  char* base = static_cast<char*>(scratch);
  // host schedules of both passes, uploaded together
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
  const int rows = uni_rows(lpt_for(n));
  const int nCB = (H + rows - 1) / rows;
  int* progress = reinterpret_cast<int*>(base + L.progress);
  cudaMemsetAsync(progress, 0, (size_t)(nCB + 2) * 4 * 2, s);
  UniArgs a;
  std::memset(&a, 0, sizeof a);
  a.W = W; a.H = H; a.n = n; a.T = T; a.nCB = nCB;
  a.raw = raw; a.agg = agg; a.depth = depth; a.planes = g.planes; a.guidance = g.guidance;
  a.p1 = p1;
  volatile float p1f = (float)p1;
  a.p2base = p1f * p2scale;
  for (int i = 0; i < 4; i++) a.gw[i] = gw[i];
  a.bnd = reinterpret_cast<uint16_t*>(base + L.bnd);
  a.bnd_min = reinterpret_cast<uint16_t*>(base + L.bnd_min);
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
  const int lpt = lpt_for(n);
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
    a.p2t = reinterpret_cast<const uint2*>(base + L.p2t);
    k_p2_table<<<dim3((W + 127) / 128, H), 128, 0, s>>>(a, reinterpret_cast<uint2*>(base + L.p2t));
    count_launches(1);
    if (lpt == 2) launch_pass<2>(a, s);
    else if (lpt == 4) launch_pass<4>(a, s);
    else if (lpt == 8) launch_pass<8>(a, s);
    else if (lpt == 16) launch_pass<16>(a, s);
    else launch_pass<24>(a, s);
    if (pass == 0 && agg_pass1) cudaMemcpyAsync(agg_pass1, agg, (size_t)W * H * n * 2, cudaMemcpyDeviceToDevice, s);
  }
  k_wta_column<<<(H * 32 + 255) / 256, 256, 0, s>>>(agg, W, H, n, 0, g.planes, depth);
  count_launches(1);
  return 0;
}

}  // namespace lux
