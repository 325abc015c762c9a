// Exact replay of DenseLayer.Compute's aggregation (DenseStereoSgm.cs:206-224) on the reference's own line-buffer layout.
//
// The reference's result depends on its traversal, not only on the SGM recurrence: sheared T-wide tiles visit the last
// column twice per band in pass +1 (column 0 in pass -1), ragged per-pixel plane ranges spill across path blocks, reads
// past a block see whatever the flat buffer holds there, and pass -1 starts from the state pass +1 left. This kernel
// keeps the flat buffer (2 halves x (W+2) slots x (4·MaxHi+5) u16, plus Min/RangeS/RangeC/Pix) in global memory and runs
// every Pixel() call of the reference in an order that gives each read the same last writer:
//   * a band of T >= 4 rows runs on blocks (parts) of min(8, T/2) rows, a warp per row (one block below); blocks take
//     tickets in order, so a part only ever waits on a running one;
//   * a part runs its tiles in order (a block barrier between tiles); inside a tile, row r runs its offset u (pixel
//     column iT - r + u) once row r-1 has finished offset u, and a part's first row follows the part above's last row:
//     at the same tile and offset within a band, at offset u of tile i+1 across bands (the same sheared frame);
//   * two calls touch a common element only when at most two columns apart, and the one pair this leaves unordered,
//     the upper row's pixel two columns right of the lower one, touches nothing in common (see the row hand-over);
//   * the revisits of the last column do not follow the sheared columns: all of a band's revisits lie at offset 0 of its
//     last tile, and the next band's first part waits for that offset before a tile that reaches column W-3; a part
//     whose rows revisit in tile i first waits for the band's last part to finish tile i-1 (a band's tiles come in order
//     in the reference);
//   * tiles taller than the flag rows step with a block barrier instead, pixel (r, u) at step u + 2r (pixels of one step
//     are three or more columns apart), one block per band, three tiles behind the band above.
// tests/test_replay_schedule_cpu.py checks these waits against the reference's order as a happens-before model.
// Within a Pixel() call a warp handles the lanes, with all of the call's line-buffer reads in one batch where its windows
// allow. The four paths run in order (a path may spill into the next), or at once on four groups of eight lanes where
// no window of the call leaves its block.
#include "common.cuh"
#include "internal.h"

namespace lux {

struct EmuArgs {
  int W, H, T, dir, xsw, min_lo, max_hi, slot_stride, halfL, halfM, halfR, gwN, ghN;
  int parts, part_rows;  // blocks per band and rows per block
  int Llen;  // line-buffer elements; the host keeps it below 2^31 - 2^16, so every index of it fits 32 bits
  uint16_t* L;
  uint16_t* Min;
  uint16_t* RangeS;
  uint16_t* RangeC;
  float4* Pix;
  const uchar4* guidance;
  const uint8_t* skip;
  const uint16_t* start;
  const uint16_t* count;
  const uint16_t* cap;
  const uint64_t* off;
  const uint8_t* raw;
  uint16_t* agg;
  int p1;
  float p2base;
  float gw[4];
  int* ticket;
  int* progress;
  int* err;
  unsigned long long timeout_ns;
  int stall_block;  // failure-path tests: this part's waits on the part above read `never` (-1: none)
  const int* never;
};

LUX_DEV int rd(const EmuArgs& a, int i) {  // Rd (DenseStereoSgm.cs:324)
  return i < 0 ? 2000 : i < a.Llen ? (int)__ldcg(a.L + i) : 0;
}

// One path of a Pixel() call (:276-314) over its cap planes, a lane per plane, each index through Rd's bounds and each
// write checked: the form for windows that reach past the buffer. Returns the lane's running minimum.
LUX_DEV int emu_path_checked(const EmuArgs& a, int nb, int baseCur, int q, int cap, int count, bool skipped,
                             const uint8_t* rawp, uint16_t* aggp, int P2p, int minPrev, int lane) {
  int runMin = 0xffff;
  for (int k = lane; k < cap; k += 32) {
    const int qi = q + k;
    const int Lm = rd(a, nb + qi - 1), L0 = rd(a, nb + qi), Lp = rd(a, nb + qi + 1);
    const int m = min(min(min(Lm + a.p1, 65535), L0), min(min(Lp + a.p1, 65535), P2p));
    const int rv = skipped ? (k < count ? 0 : 255) : rawp[k];
    int lc = min(rv + m, 65535) - minPrev;
    if (lc < 0) lc = 0;
    const int wi = baseCur + qi;
    if (wi < 0 || wi >= a.Llen) atomicCAS(a.err, 0, 7);
    else __stcg(a.L + wi, (uint16_t)lc);
    runMin = min(runMin, lc);
    aggp[k] = (uint16_t)min((int)aggp[k] + lc, 65535);
  }
  return runMin;
}

// The same path where the read window Ln[-1 .. cap] and the write window Lw[0 .. cap) lie inside the buffer and do not
// meet: KB iterations of the lanes have their loads issued before their stores, one L2 round trip per batch. Caps are
// multiples of 8 here (checked before the launch).
template <int KB>
LUX_DEV int emu_path_batched(const uint16_t* Ln, uint16_t* Lw, int p1, int cap, int count, bool skipped, const uint8_t* rawp,
                             uint16_t* aggp, int P2p, int minPrev, int lane) {
  int runMin = 0xffff;
  for (int k0 = lane; k0 < cap; k0 += 32 * KB) {
    int Lm[KB], L0[KB], Lp[KB], rv[KB], ag[KB];
#pragma unroll
    for (int u = 0; u < KB; u++) {
      const int k = k0 + 32 * u;
      if (k < cap) {
        Lm[u] = __ldcg(Ln + k - 1);
        L0[u] = __ldcg(Ln + k);
        Lp[u] = __ldcg(Ln + k + 1);
        rv[u] = skipped ? (k < count ? 0 : 255) : rawp[k];
        ag[u] = aggp[k];
      }
    }
#pragma unroll
    for (int u = 0; u < KB; u++) {
      const int k = k0 + 32 * u;
      if (k >= cap) break;
      const int m = min(min(min(Lm[u] + p1, 65535), L0[u]), min(min(Lp[u] + p1, 65535), P2p));
      int lc = min(rv[u] + m, 65535) - minPrev;
      if (lc < 0) lc = 0;
      __stcg(Lw + k, (uint16_t)lc);
      runMin = min(runMin, lc);
      aggp[k] = (uint16_t)min(ag[u] + lc, 65535);
    }
  }
  return runMin;
}

// The forms below take a Pixel() call's line-buffer reads in one batch, issued together with its line state, and make
// each plane's three neighbours (window elements k-1, k, k+1) from one load per element by shuffles. R holds the batch in
// registers (compile-time indices only).

// Plane k's window neighbours from the lanes of a segment of `width` lanes: element e of the window sits in chunk
// (e + 1) / width at lane (e + 1) % width, so lane i of chunk c holds element c·width + i - 1, its own Lm.
template <int width>
LUX_DEV void emu_neighbours(int x0, int x1, int i, int& L0, int& Lp) {
  const int d1 = __shfl_down_sync(0xffffffffu, x0, 1, width), d2 = __shfl_down_sync(0xffffffffu, x0, 2, width);
  const int n0 = __shfl_sync(0xffffffffu, x1, 0, width), n1 = __shfl_sync(0xffffffffu, x1, 1, width);
  L0 = i < width - 1 ? d1 : n0;
  Lp = i < width - 2 ? d2 : i == width - 2 ? n0 : n1;
}

// The grouped form in one batch (cap <= 8·KBG): lane j of group grp holds elements 8u + j - 1 of path grp's read window
// Ln[-1 .. cap] in R[u] (u = 0..KBG), the raw costs of planes 8u + j in R[KBG + 1 + u] and (group 0) their aggregates in
// R[2·KBG + 1 + u].
template <int KBG, int NR>
LUX_DEV void emu_group_load1(const uint16_t* Ln, int cap, int count, bool skipped, const uint8_t* rawp, const uint16_t* aggp,
                             int j, int grp, int (&R)[NR]) {
  static_assert(3 * KBG + 1 <= NR, "register batch too small");
#pragma unroll
  for (int u = 0; u <= KBG; u++) {
    const int e = 8 * u + j - 1;
    R[u] = e <= cap ? (int)__ldcg(Ln + e) : 0;
  }
#pragma unroll
  for (int u = 0; u < KBG; u++) {
    const int k = 8 * u + j;
    R[KBG + 1 + u] = k < cap ? (skipped ? (k < count ? 0 : 255) : (int)rawp[k]) : 0;
    R[2 * KBG + 1 + u] = k < cap && grp == 0 ? (int)aggp[k] : 0;
  }
}

// The four paths of a Pixel() call at once, lanes 8p..8p+7 on path p, from the batch emu_group_load1 loaded, where every
// write and cleanup window of the call lies inside its own block (q + cap and q0 + cp at most MaxHi + 1) and every read
// inside the buffer. Then no path reads what another writes (the reads are neighbour slots or the other half; the writes
// are this slot's four blocks), so the paths may run together, and the cleanup need only write the part of the old range
// the new one does not overwrite. The aggregate takes the four paths' sum at once: saturating adds of non-negative terms
// commute, min(min(a + x, C) + y, C) = min(a + x + y, C). Caps are multiples of 8 here (checked before the launch), so
// every lane of a chunk has a plane.
template <int KBG, int NR>
LUX_DEV void emu_pixel_grouped1(const EmuArgs& a, int baseCur, int q, int q0, int cap, int cp, uint16_t* aggp,
                                int P2p, int minPrev, uint16_t* minOut, int lane, const int (&R)[NR]) {
  const int j = lane & 7, grp = lane >> 3;
  for (int k = (q0 < 0 ? -q0 : 0) + j; k < cp; k += 8) {  // stale cleanup (:261-263), outside the new range
    const int idx = q0 + k;
    if (idx < q || idx >= q + cap) __stcg(a.L + baseCur + idx, (uint16_t)2000);
  }
  uint16_t* Lw = a.L + (baseCur + q);
  int runMin = 0xffff;
#pragma unroll
  for (int u = 0; u < KBG; u++) {
    if (8 * u >= cap) break;  // warp-uniform: the cap is the pixel's
    const int k = 8 * u + j;
    int L0, Lp;
    emu_neighbours<8>(R[u], R[u + 1], j, L0, Lp);
    const int m = min(min(min(R[u] + a.p1, 65535), L0), min(min(Lp + a.p1, 65535), P2p));
    int lc = min(R[KBG + 1 + u] + m, 65535) - minPrev;
    if (lc < 0) lc = 0;
    __stcg(Lw + k, (uint16_t)lc);
    runMin = min(runMin, lc);
    int sum = lc + __shfl_xor_sync(0xffffffffu, lc, 8);
    sum += __shfl_xor_sync(0xffffffffu, sum, 16);
    if (grp == 0) aggp[k] = (uint16_t)min(R[2 * KBG + 1 + u] + sum, 65535);
  }
  runMin = min(runMin, __shfl_xor_sync(0xffffffffu, runMin, 1));
  runMin = min(runMin, __shfl_xor_sync(0xffffffffu, runMin, 2));
  runMin = min(runMin, __shfl_xor_sync(0xffffffffu, runMin, 4));
  if (j == 0) __stcg(minOut, (uint16_t)runMin);
}

// The path-serial form in one batch (cap <= 32·CH - 2): R[p·CH + c] holds element 32c + lane - 1 of path p's read window
// Ln_p[-1 .. cap], R[4·CH + c] the raw cost and R[5·CH + c] the aggregate of plane 32c + lane.
template <int CH, int NR>
LUX_DEV void emu_serial_load1(const uint16_t* L, const int (&win)[4], int cap, int count, bool skipped, const uint8_t* rawp,
                              const uint16_t* aggp, int lane, int (&R)[NR]) {
  static_assert(6 * CH <= NR, "register batch too small");
#pragma unroll
  for (int c = 0; c < CH; c++) {
    const int e = 32 * c + lane - 1;
#pragma unroll
    for (int p = 0; p < 4; p++) R[p * CH + c] = e <= cap ? (int)__ldcg(L + win[p] + e) : 0;
    const int k = 32 * c + lane;
    R[4 * CH + c] = k < cap ? (skipped ? (k < count ? 0 : 255) : (int)rawp[k]) : 0;
    R[5 * CH + c] = k < cap ? (int)aggp[k] : 0;
  }
}

// The four paths in the reference's order (a path's cleanup and writes may spill into the next block), each from its
// window in the batch. The batch went out before any of the call's writes, which reads no element earlier than the
// reference does: paths 1-3 read the other half, which the call does not write; path 0 reads the slot beside its own,
// which only path 3's spill can reach (pass -1), after path 0; and the windows stay clear of the call's own slot (checked
// by the caller: q + cap + 2 <= slot stride). The aggregate takes the four paths' sum at once (saturating adds of
// non-negative terms commute).
template <int CH, int NR>
LUX_DEV void emu_pixel_serial1(const EmuArgs& a, int cur, int slot, int q, int sp, int cp, int cap, uint16_t* aggp,
                               int gMinPrev, int gP2, int lane, int (&R)[NR]) {
#pragma unroll
  for (int p = 0; p < 4; p++) {
    const int baseCur = (int)cur * a.halfL + (int)slot * a.slot_stride + 1 + (int)p * (a.max_hi + 1);
    {  // stale cleanup of the previously stored range (:261-263)
      const int q0 = sp - a.min_lo, k0 = q0 < 0 ? -q0 : 0;
      const int k1 = min((int)cp, a.Llen - baseCur - q0);
      for (int k = k0 + lane; k < k1; k += 32) __stcg(a.L + baseCur + q0 + k, (uint16_t)2000);
    }
    __syncwarp();
    const int minPrev = __shfl_sync(0xffffffffu, gMinPrev, 8 * p), P2 = __shfl_sync(0xffffffffu, gP2, 8 * p);
    const int P2p = min(P2 + minPrev, 65535);
    uint16_t* Lw = a.L + (baseCur + q);
    int runMin = 0xffff;
#pragma unroll
    for (int c = 0; c < CH; c++) {
      if (32 * c >= cap) break;  // warp-uniform
      const int k = 32 * c + lane;
      const int x0 = R[p * CH + c];
      int L0, Lp;
      emu_neighbours<32>(x0, R[p * CH + (c + 1 < CH ? c + 1 : c)], lane, L0, Lp);  // chunk CH-1's lanes 30, 31 have no plane
      const int m = min(min(min(x0 + a.p1, 65535), L0), min(min(Lp + a.p1, 65535), P2p));
      int lc = min(R[4 * CH + c] + m, 65535) - minPrev;
      if (lc < 0) lc = 0;
      if (k < cap) {
        __stcg(Lw + k, (uint16_t)lc);
        runMin = min(runMin, lc);
        R[5 * CH + c] += lc;
      }
    }
    runMin = __reduce_min_sync(0xffffffffu, (unsigned)runMin);
    __syncwarp();  // this path's stores (a spill reaches the next block) before the next path's cleanup
    if (lane == 0) __stcg(a.Min + cur * a.halfM + slot * 4 + p, (uint16_t)runMin);
  }
#pragma unroll
  for (int c = 0; c < CH; c++) {
    const int k = 32 * c + lane;
    if (k < cap) aggp[k] = (uint16_t)min(R[5 * CH + c], 65535);
  }
}

// A pixel's read-only inputs, loaded before the hand-over that lets it run.
struct EmuPix {
  uchar4 gb;
  int start, count, cap, skip;
  unsigned long long off;
};
LUX_DEV EmuPix emu_load_pix(const EmuArgs& a, int x, int y) {
  const int pi = y * a.W + x;
  EmuPix s;
  s.gb = a.guidance[pi];
  s.start = a.start[pi];
  s.count = a.count[pi];
  s.cap = a.cap[pi];
  s.skip = a.skip[pi];
  s.off = a.off[pi];
  return s;
}

// Pixel (DenseStereoSgm.cs:234-317), one warp. The line-state loads (own Range, neighbours' Min and Pix) and, where the
// windows allow, every line-buffer read of the call go out as one batch: the grouped form for caps up to 8·KBG, the
// path-serial form for caps up to 32·CH - 2. Otherwise (larger caps, windows at the buffer's ends) the paths run one at
// a time below, KB iterations of a path's plane loop sharing one L2 round trip.
template <int KB, int KBG, int CH>
LUX_DEV void emu_pixel(const EmuArgs& a, int x, const EmuPix& px, int cur, int other, int lane) {
  constexpr int NR = 6 * CH > 3 * KBG + 1 ? 6 * CH : 3 * KBG + 1;
  const int slot = x + 1;
  const int start = px.start, count = px.count, cap = px.cap;
  const bool skipped = px.skip != 0;
  const uint8_t* rawp = a.raw + px.off;
  uint16_t* aggp = a.agg + px.off;
  const int sp = __ldcg(a.RangeS + cur * a.halfR + slot), cp = __ldcg(a.RangeC + cur * a.halfR + slot);
  // Lanes 8p..8p+7 read path p's neighbour Min and Pix entries and make its P2 up front: this call writes only its own
  // slot of the current half, and every entry read here is another slot or the other half.
  const int gp = lane >> 3;
  const int gns = slot + (gp == 2 ? 0 : gp == 3 ? a.dir : -a.dir);
  const int ghalf = gp == 0 ? cur : other;
  const int gMinPrev = __ldcg(a.Min + ghalf * a.halfM + gns * 4 + gp);
  const float4 pn4 = __ldcg(a.Pix + ghalf * a.halfR + gns);
  const int q = start - a.min_lo;
  const int gnb = (int)ghalf * a.halfL + (int)gns * a.slot_stride + 1 + (int)gp * (a.max_hi + 1);
  // The grouped form needs every write window inside its own block and every read inside the buffer (checked here) and
  // the cleanup window inside its block (checked once the Range entries are in). The path-serial batch needs its four
  // read windows and write ranges inside the buffer and clear of each other.
  const bool grouped = cap <= 8 * KBG && q + cap <= a.max_hi + 1 && __all_sync(0xffffffffu, gnb + q + cap + 1 <= a.Llen);
  bool serial = false;
  int win[4];
  if (!grouped) {
    const int own = (int)cur * a.halfL + (int)slot * a.slot_stride + 1;
    serial = cap <= 32 * CH - 2 && q + cap + 2 <= a.slot_stride;
#pragma unroll
    for (int p = 0; p < 4; p++) {
      const int ns = slot + (p == 2 ? 0 : p == 3 ? a.dir : -a.dir);
      const int nb = (int)(p == 0 ? cur : other) * a.halfL + (int)ns * a.slot_stride + 1 + (int)p * (a.max_hi + 1);
      const int wb = own + (int)p * (a.max_hi + 1) + q;
      win[p] = nb + q;
      serial = serial && nb + q - 1 >= 0 && nb + q + cap + 1 <= a.Llen && wb >= 0 && wb + cap <= a.Llen;
    }
  }
  int R[NR];
  if (grouped) emu_group_load1<KBG>(a.L + (gnb + q), cap, count, skipped, rawp, aggp, lane & 7, gp, R);
  else if (serial) emu_serial_load1<CH>(a.L, win, cap, count, skipped, rawp, aggp, lane, R);
  const float g[4] = {(float)px.gb.x, (float)px.gb.y, (float)px.gb.z, (float)px.gb.w};
  if (lane == 0) __stcg(a.Pix + cur * a.halfR + slot, make_float4(g[0], g[1], g[2], g[3]));
  int gP2;
  {
    const float pn[4] = {pn4.x, pn4.y, pn4.z, pn4.w};
    gP2 = sgm_p2(g, pn, a.gw, a.p2base);
  }
  bool done = false;
  if (grouped) {
    const int q0 = sp - a.min_lo;
    if (cp == 0 || q0 + cp <= a.max_hi + 1) {
      const int gbase = (int)cur * a.halfL + (int)slot * a.slot_stride + 1 + (int)gp * (a.max_hi + 1);
      emu_pixel_grouped1<KBG>(a, gbase, q, q0, cap, cp, aggp, min(gP2 + gMinPrev, 65535), gMinPrev,
                              a.Min + cur * a.halfM + slot * 4 + gp, lane, R);
      done = true;
    }
  } else if (serial) {
    emu_pixel_serial1<CH>(a, cur, slot, q, sp, cp, cap, aggp, gMinPrev, gP2, lane, R);
    done = true;
  }
  if (done) {
    if (lane == 0) {
      __stcg(a.RangeS + cur * a.halfR + slot, (uint16_t)start);
      __stcg(a.RangeC + cur * a.halfR + slot, (uint16_t)cap);
    }
    __syncwarp();
    return;
  }
#pragma unroll 1
  for (int p = 0; p < 4; p++) {
    const int baseCur = (int)cur * a.halfL + (int)slot * a.slot_stride + 1 + (int)p * (a.max_hi + 1);
    {  // stale cleanup of the previously stored range (:261-263)
      int q0 = sp - a.min_lo, k0 = q0 < 0 ? -q0 : 0;
      int k1 = min((int)cp, a.Llen - baseCur - q0);
      for (int k = k0 + lane; k < k1; k += 32) __stcg(a.L + baseCur + q0 + k, (uint16_t)2000);
    }
    __syncwarp();
    const int ns = slot + (p == 2 ? 0 : p == 3 ? a.dir : -a.dir);
    const int half = p == 0 ? cur : other;
    const int minPrev = __shfl_sync(0xffffffffu, gMinPrev, 8 * p), P2 = __shfl_sync(0xffffffffu, gP2, 8 * p);
    const int P2p = min(P2 + minPrev, 65535);
    if (cap == 0) {
      __syncwarp();
      if (lane == 0) __stcg(a.Min + cur * a.halfM + slot * 4 + p, (uint16_t)0xffff);
      __syncwarp();
      continue;
    }
    const int nb = (int)half * a.halfL + (int)ns * a.slot_stride + 1 + (int)p * (a.max_hi + 1);
    const int q = start - a.min_lo;
    // A path reads L[nb + q - 1 .. nb + q + cap] and writes L[baseCur + q .. baseCur + q + cap - 1]. The bases lie a
    // whole half apart (paths 1-3) or one slot stride apart (path 0), so the windows meet only if cap + 2 exceeds the
    // slot stride (4·MaxHi + 5). Where they stay apart and inside the buffer, the batched form runs; otherwise one plane
    // per lane step with every index checked, reading and writing in the reference's order.
    const bool batched = cap + 2 <= a.slot_stride && nb + q - 1 >= 0 && nb + q + cap + 1 <= a.Llen && baseCur + q >= 0 &&
                         baseCur + q + cap <= a.Llen;
    int runMin = batched ? emu_path_batched<KB>(a.L + (nb + q), a.L + (baseCur + q), a.p1, cap, count, skipped, rawp, aggp, P2p,
                                                minPrev, lane)
                         : emu_path_checked(a, nb, baseCur, q, cap, count, skipped, rawp, aggp, P2p, minPrev, lane);
    runMin = __reduce_min_sync(0xffffffffu, (unsigned)runMin);
    __syncwarp();  // this path's stores (a spill reaches the next block) before the next path's cleanup
    // No lane of this call reads its own Min entry; the next reader runs after the step's __syncthreads.
    if (lane == 0) __stcg(a.Min + cur * a.halfM + slot * 4 + p, (uint16_t)runMin);
  }
  if (lane == 0) {
    __stcg(a.RangeS + cur * a.halfR + slot, (uint16_t)start);
    __stcg(a.RangeC + cur * a.halfR + slot, (uint16_t)cap);
  }
  __syncwarp();
}

// The tile's pixel (row r, xp offset u) of a band: x, y and whether there is one. The clamped row start revisits the
// last column at u = 0 only.
struct EmuTileRow {
  int yp, xs, xe;
  bool revisit;
};
LUX_DEV EmuTileRow emu_tile_row(const EmuArgs& a, int j, int i, int r) {
  EmuTileRow t;
  t.yp = j * a.T + r;
  t.xs = min(max(i * a.T - r, 0), (a.xsw && a.dir > 0) ? a.W : a.W - 1);
  t.xe = min(max(i * a.T + a.T - r, -1), a.W);
  t.revisit = i * a.T - r >= a.W;
  return t;
}
LUX_DEV bool emu_tile_pixel(const EmuArgs& a, const EmuTileRow& t, int i, int r, int u, int& x, int& y) {
  if (t.yp >= a.H || t.xs == t.xe) return false;  // yEnd (:213); an empty row range
  int xp;
  if (t.revisit) {
    if (u != 0) return false;
    xp = a.W - 1;
  } else {
    xp = i * a.T - r + u;
    if (xp < t.xs || xp >= t.xe) return false;
  }
  x = a.dir > 0 ? xp : a.W - 1 - xp;
  y = a.dir > 0 ? t.yp : a.H - 1 - t.yp;
  return true;
}

constexpr int kFlagRows = 64;  // tiles up to this many rows hand over row to row (a warp a row); taller ones step with a barrier

// kThreads bounds the block and with it the registers a thread may hold for a Pixel() call's batch: 256 for the row form
// (parts of at most 8 rows; caps up to 574 planes in one batch, the plane counts of the whole L16 pyramid), 1024 for
// the barrier form. KB, KBG, CH: emu_pixel's batch sizes. kFlags: the row hand-over below (even T <= kFlagRows), else a
// barrier per step of the sheared schedule, pixel (r, u) at step u + 2r (pixels of one step are three or more columns
// apart).
//
//
// Each warp owns one row of its part and runs the row's offsets u in order through all tiles; row r runs offset u of a
// tile once row r-1 has finished offset u (a CTA-scope release/acquire of the row's count in shared memory): the
// recurrence reads row r-1 at columns x-1, x and x+1, offsets u-2..u. For rows r1 < r2 this orders (r1, u1) before
// (r2, u2) whenever u1 <= u2. Two pixels touch a common element only when at most two columns apart, x1 - x2 =
// (r2 - r1) + (u1 - u2) <= 2, so the one pair left unordered is the upper row's pixel two columns right of the lower
// one (r2 = r1 + 1, u1 = u2 + 1), and it touches nothing in common:
//   * the lower pixel reads the upper row's half at columns x2-1..x2+1 (each block window +-1 element) and, past its
//     path-3 window, the pad element of the next slot in memory; the upper pixel writes its own blocks (never its own
//     pad) and spills at most align - 2 <= 6 elements (q + cap <= MaxHi - MinLo + align - 1) into the pad and first
//     block-0 elements of its next slot in memory, which is column x2 + 3 (pass +1) or x2 + 1 (pass -1), where the lower
//     pixel reads only block 3 from index -1 (block 2's last);
//   * the lower pixel writes the other half, which the upper pixel reads at columns x2+1..x2+3: its spill (pass +1)
//     reaches slot x2+1's pad and block-0 elements 0..5, and the upper pixel reads that slot's block 1 from index -1,
//     block 0's last element (index MaxHi >= 8 with align 8; with align 2 nothing spills).
// Rows then advance at their own pace, one pixel apart, instead of two pixels apart with each step waiting for its
// slowest pixel.
template <int kThreads, int KB, int KBG, int CH, bool kFlags>
__global__ void __launch_bounds__(kThreads) k_sgm_emulate(const EmuArgs a) {
  __shared__ int s_part;
  __shared__ volatile int s_stop;
  __shared__ int s_row[kFlagRows];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  if (tid == 0) {
    s_part = atomicAdd(a.ticket, 1);
    s_stop = 0;
  }
  __syncthreads();
  const int k = s_part;  // tickets in order: the part above (k - 1) is running or done
  const int j = k / a.parts, part = k % a.parts;
  const int T = a.T;
  if (j >= a.ghN) return;
  const int r0 = part * a.part_rows, r1 = min(r0 + a.part_rows, T);  // this part's rows of the tile frame
  // A part below the image has no pixels, and neither has any part after it: nothing waits on its progress. (It must
  // not wait either: the last row of the part above, below the image too, publishes none.)
  if (j * T + r0 >= a.H) return;
  int* const above = k == a.stall_block ? const_cast<int*>(a.never) : a.progress + (k - 1);  // the part above: its last row's offsets
  if constexpr (kFlags) {
    // One row per warp; s_row[r] counts row r's offsets done across tiles (i·T + u + 1). A row goes on into the next
    // tile by itself: the only pixels of a later tile that lower rows' earlier tiles can touch are revisits of the
    // last column, and a row waits for its part's last row to finish tile i-1 before revisiting in tile i.
    for (int r = tid; r < kFlagRows; r += blockDim.x) s_row[r] = 0;
    __syncthreads();
    const int r = r0 + warp;
    if (r >= r1) return;
    const int r_pub = min(r1, a.H - j * T) - 1;  // the part's last row inside the image, which publishes
    if (j * T + r >= a.H) {                       // past the image: no pixels, and only rows past it wait on it
      if (lane == 0) st_release_cta(&s_row[r], 0x7fffffff);
      return;
    }
    const bool publish = r == r_pub;
    int seen = 0;  // first row: the part above's last-row offsets seen so far
    for (int i = 0; i < a.gwN; i++) {
      const EmuTileRow row = emu_tile_row(a, j, i, r);
      // Another block reads what this part's last two rows write (the row above it in the other half, the row two
      // above in its own half: the Range entries of its stale cleanup, the line state it overwrites), and, on a tile
      // before the part above revisits, what any row writes near the last column. No fence is needed for that: every
      // hand-over is a release / acquire pair (a row's lanes __syncwarp, lane 0 releases its count at CTA scope, the
      // next row's lanes acquire it; the publishing row releases at GPU scope, the next block's lanes acquire), so a
      // write of any row is ordered, through the chain of hand-overs, before every read that waits on it (the PTX
      // memory model's causality order is transitive across the CTA- and GPU-scope links).
      // Waits at the tile's start, around revisits of the last column (which do not follow the sheared columns):
      // the first part's first row waits, before a tile that reaches column W-3 (whose calls touch the last column's
      // slots), for the band above's revisits: offset 0 of its last tile, where all of them lie (the band above comes
      // first in the reference); a first row whose part revisits in tile i waits for the band's last part (and so
      // every part below it) to finish tile i-1, and any revisiting row for its own part's last row (a band's tiles
      // come in order in the reference).
      int gneed = 0;
      int* gflag = above;
      if (r == r0 && part == 0 && k > 0 && (i + 1) * T >= a.W - 2) gneed = (a.gwN - 1) * T + 1;
      const int last = min(a.parts - 1, (a.H - j * T - 1) / a.part_rows);  // the band's last part inside the image
      if (r == r0 && part < last && i > 0 && i * T - r0 >= a.W) {
        gneed = i * T;  // (a first part's row r0 revisiting at tile i has no tile i+2 wait: i * T >= W)
        gflag = a.progress + ((size_t)j * a.parts + last);
      }
      bool failed = false;
      if (gneed > 0 && __reduce_min_sync(0xffffffffu, wait_at_least_value(gflag, gneed, a.err, 11, a.timeout_ns)) < 0) {
        failed = true;
      } else if (i > 0 && i * T - r >= a.W && r != r_pub &&
                 __any_sync(0xffffffffu, !wait_shared_at_least(&s_row[r_pub], i * T, &s_stop, a.timeout_ns))) {
        failed = true;
      }
      if (failed) {
        if (lane == 0) {
          atomicCAS(a.err, 0, 11);  // LUX_ERR_TIMEOUT, or another warp's failure
          s_stop = 1;
        }
        return;
      }
      int nx, ny;
      bool has_next = emu_tile_pixel(a, row, i, r, 0, nx, ny);
      EmuPix next;
      if (has_next) next = emu_load_pix(a, nx, ny);
      for (int u = 0; u < T; u++) {
        const bool has = has_next;
        const int x = nx;
        const EmuPix px = next;
        // The next offset's read-only inputs, loaded while this offset waits and runs.
        has_next = u + 1 < T && emu_tile_pixel(a, row, i, r, u + 1, nx, ny);
        if (has_next) next = emu_load_pix(a, nx, ny);
        if (r > r0 && __any_sync(0xffffffffu, !wait_shared_at_least(&s_row[r - 1], i * T + u + 1, &s_stop, a.timeout_ns))) {
          if (lane == 0) {
            atomicCAS(a.err, 0, 11);
            s_stop = 1;
          }
          return;
        }
        // The first row continues the part above's last row one row down: within the band, that row at the same
        // tile and offset; across bands, the band above's last row at offset u of tile i+1 (the same sheared frame).
        if (r == r0 && k > 0) {
          const int target = part > 0 ? i * T + u + 1 : min((i + 1) * T + u + 1, a.gwN * T);
          if (seen < target) {
            seen = __reduce_min_sync(0xffffffffu, wait_at_least_value(above, target, a.err, 11, a.timeout_ns));
            if (seen < 0) {
              if (lane == 0) s_stop = 1;
              return;
            }
          }
        }
        if (has) {
          const int cur = (r & 1) == 0 ? 1 : 0;
          emu_pixel<KB, KBG, CH>(a, x, px, cur, 1 - cur, lane);
        }
        __syncwarp();
        if (lane == 0) {
          st_release_cta(&s_row[r], i * T + u + 1);
          if (publish) st_release(a.progress + k, i * T + u + 1);  // all rows above it are through u as well
        }
      }
    }
  } else {
  // Tiles taller than the flag rows: a block barrier per step of the sheared schedule, three tiles behind the band
  // above (progress counts tiles times T).
  for (int i = 0; i < a.gwN; i++) {
    if (tid == 0) {
      if (k > 0 && !wait_at_least(above, min(i + 3, a.gwN) * T, a.err, 11 /* LUX_ERR_TIMEOUT */, a.timeout_ns)) s_stop = 1;
      if (*(volatile int*)a.err != 0) s_stop = 1;
    }
    __syncthreads();
    if (s_stop) break;
    for (int t = 0; t <= 3 * T - 3; t++) {
      const int rlo = max(0, (t - T + 2) / 2), rhi = min(T - 1, t / 2);
      for (int r = rlo + warp; r <= rhi; r += nw) {
        const int u = t - 2 * r;
        const EmuTileRow row = emu_tile_row(a, j, i, r);
        int x, y;
        if (!emu_tile_pixel(a, row, i, r, u, x, y)) continue;
        const int cur = (r & 1) == 0 ? 1 : 0;
        emu_pixel<KB, KBG, CH>(a, x, emu_load_pix(a, x, y), cur, 1 - cur, lane);
      }
      __syncthreads();
    }
    __syncthreads();
    if (s_stop) break;
    if (tid == 0) {
      __threadfence();
      st_release(a.progress + k, (i + 1) * T);
    }
  }
  }
}

size_t emu_line_buffer_elems(int W, int max_hi) { return (size_t)2 * (W + 2) * (4 * (size_t)max_hi + 5); }

__global__ void k_emu_init(uint16_t* Min, uint16_t* RangeS, uint16_t* RangeC, float4* Pix, int slots, int align) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 2 * slots * 4) Min[i] = 2000;
  if (i < 2 * slots) {
    RangeS[i] = 0;
    RangeC[i] = (uint16_t)align;
    Pix[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

void emu_init_buffers(const EmuBuffers& b, int W, int max_hi, int align, int bands, cudaStream_t s) {
  launch_fill_u16(b.L, b.Llen, 2000, s);  // AllocLineBuffers (DenseStereoSgm.cs:158-165)
  int slots = W + 2;
  k_emu_init<<<(2 * slots * 4 + 255) / 256, 256, 0, s>>>(b.Min, b.RangeS, b.RangeC, b.Pix, slots, align);
  count_launches(1);
  cudaMemsetAsync(b.ticket, 0, 2 * sizeof(int), s);
  cudaMemsetAsync(b.progress, 0, (size_t)2 * bands * kEmuParts * sizeof(int), s);
}

void launch_sgm_emulate(const LayerGeom& g, const EmuBuffers& b, int dir, int xsw, uint16_t p1, float p2scale, const float gw[4],
                        const uint8_t* raw, uint16_t* agg, int* err, cudaStream_t s) {
  EmuArgs a;
  a.W = g.W; a.H = g.H; a.T = g.tile; a.dir = dir; a.xsw = xsw;
  a.min_lo = g.min_lo; a.max_hi = g.max_hi;
  a.slot_stride = 4 * g.max_hi + 5;
  a.halfL = (g.W + 2) * a.slot_stride;
  a.halfM = (g.W + 2) * 4;
  a.halfR = g.W + 2;
  a.gwN = (g.W + 2 * g.tile - 1) / g.tile;
  a.ghN = (g.H + g.tile - 1) / g.tile;
  a.Llen = (int)b.Llen;
  a.L = b.L; a.Min = b.Min; a.RangeS = b.RangeS; a.RangeC = b.RangeC; a.Pix = b.Pix;
  a.guidance = g.guidance; a.skip = g.skip; a.start = g.start; a.count = g.count; a.cap = g.cap; a.off = g.off;
  a.raw = raw; a.agg = agg;
  a.p1 = p1;
  volatile float p1f = (float)p1;
  a.p2base = p1f * p2scale;  // (float)P1 * P2Scale (:256)
  for (int i = 0; i < 4; i++) a.gw[i] = gw[i];
  int pass = dir > 0 ? 0 : 1;
  // The row form splits a band of T >= 4 rows between blocks (parts) of min(8, T/2) rows, a warp a row (up to 8 warps
  // a block, so that a thread may hold a whole Pixel() call's batch; shorter parts also spread a band over more SMs,
  // which measured faster than 16-row parts on every L16 layer). It needs an even T: the line-buffer half of a row
  // follows its row in the tile (as in the reference), so with an odd T a band's last row and the next band's first
  // row share a half, and the pair two columns apart that the row form leaves unordered would then meet (the upper
  // pixel's path-0 read of the slot the lower one spills into).
  const bool flags = g.tile <= kFlagRows && g.tile % 2 == 0;
  a.part_rows = flags && g.tile >= 4 ? min(kEmuPartRows, g.tile / 2) : g.tile;
  a.parts = (g.tile + a.part_rows - 1) / a.part_rows;  // at most kEmuParts (T <= kFlagRows = 64)
  a.ticket = b.ticket + pass;
  a.progress = b.progress + (size_t)pass * a.ghN * kEmuParts;
  a.err = err;
  a.timeout_ns = g.timeout_ns;
  a.stall_block = g.stall_block;
  a.never = g.never;
  int nw = flags ? a.part_rows : g.tile / 2;
  if (nw < 1) nw = 1;
  if (nw > 32) nw = 32;
  const int blocks = a.ghN * a.parts;
  if (!flags) k_sgm_emulate<1024, 1, 4, 2, false><<<blocks, nw * 32, 0, s>>>(a);
  else k_sgm_emulate<256, 4, 8, 18, true><<<blocks, nw * 32, 0, s>>>(a);  // nw = part_rows <= 8
  count_launches(1);
}

}  // namespace lux
