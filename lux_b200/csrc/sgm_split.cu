// Aggregation of a uniform layer by path groups (bit-exact with DenseStereoSgm.cs:181-324, like sgm_uniform.cu).
//
// The four paths of a pass read different neighbours: path 0 (x-1, y), path 1 (x-1, y-1), path 2 (x, y-1), path 3
// (x+1, y-1). Fused, they force row y to trail row y-1 by two pixels, so a pass takes (2H + W) pixel steps of one row.
// Split into two groups, each has a short critical path and thousands of independent chains:
//   group A = paths {0, 1}: a chain per row, stepping along x; all rows advance together, row y taking path 1 from
//             row y-1 at the previous step (critical path W);
//   group B = paths {2, 3}: a chain per column, stepping down y; all columns advance together, column x taking path 3
//             from column x+1 at the previous step (critical path H).
// One kernel serves both: chain j carries its own path (0 or 2) in registers and reads its neighbour path (1 or 3) of
// chain j-1 from a shared-memory ring (full / empty mbarriers, as in sgm_uniform.cu); a loader and a publisher warp
// carry chain j-1 across block boundaries through global band buffers. The aggregates are summed over the kernels in
// u16 (order-free): pass +1: A stores agg, B adds; pass -1: A adds, B adds and takes the WTA.
//
// The reference's revisits of the last column c (revisit_schedule.h) split by path too: paths 0 and 1 of a revisit read
// only normal visits of column c-1 (or the boundary), so k_revisit01 runs them as independent warps after group A;
// path 2 reads column c's own chain (normal visits and earlier revisits), so the group-B warp of column c replays its
// revisit batches in the reference's order; path 3 restarts from the margin.
#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "revisit_schedule.h"
#include "sgm_paths.cuh"

namespace lux {

namespace {

constexpr int kMaxChainWarps = 15;     // chain warps per block at most (two chains each), sized to the register file
constexpr int kMaxWarpsS = kMaxChainWarps + 2;  // plus the loader and the publisher
constexpr int kRingS = 8;              // slots of a chain's hand-over ring
constexpr int kStageS = 6;             // steps of raw costs and aggregates staged ahead per chain warp (cp.async)

struct SplitArgs {
  UniArgs u;              // layer, pass and revisit-schedule fields shared with the fused kernel
  int group;              // 0: paths {0, 1}, chains = rows; 1: paths {2, 3}, chains = columns from the right
  int nchains, nsteps;    // A: H rows of W steps; B: W columns of H steps
  // The neighbour-path state of every block's last chain, one buffer per block: a chain can run one step ahead of the
  // chain above it, so later blocks may catch up with earlier ones and a buffer cannot be reused within a launch.
  uint16_t* bnd;          // [blocks][nsteps][Dp]
  uint16_t* bnd_min;      // [blocks][nsteps]
  const int* rev_rows;    // k_revisit01: the rows with a revisit
  int n_rev;
};

// The own path (o: 0 / 2, carried by the chain) and the neighbour path (b: 1 / 3, from the chain before) of NC chains'
// pixels, all interleaved so the independent recurrences overlap. acc[k] gets both paths of chain k.
template <int LPT, bool FULL, int NC>
LUX_DEV void chain_paths(const Src<LPT> (&so)[NC], const uint32_t (&p2o)[NC], const Src<LPT> (&sb)[NC], const uint32_t (&p2b)[NC],
                         uint32_t p1x2, const V<LPT> (&raw2)[NC], bool active, int lane, V<LPT> (&outo)[NC], V<LPT> (&outb)[NC],
                         V<LPT> (&acc)[NC], uint32_t (&mino)[NC], uint32_t (&minb)[NC]) {
  constexpr int NR = LPT / 2;
  uint32_t prev[NC][2], next[NC][2], p2x[NC][2], m2[NC][2], rm[NC][2];
#pragma unroll
  for (int k = 0; k < NC; k++) {
    prev[k][0] = __shfl_up_sync(0xffffffffu, so[k].L.r[NR - 1], 1);
    next[k][0] = __shfl_down_sync(0xffffffffu, so[k].L.r[0], 1);
    prev[k][1] = __shfl_up_sync(0xffffffffu, sb[k].L.r[NR - 1], 1);
    next[k][1] = __shfl_down_sync(0xffffffffu, sb[k].L.r[0], 1);
  }
#pragma unroll
  for (int k = 0; k < NC; k++) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (lane == 0) prev[k][h] = kInit2;   // plane -1: 2000
      if (lane == 31) next[k][h] = kInit2;  // plane n (or a padding lane): 2000
      rm[k][h] = 0xffffffffu;
    }
    p2x[k][0] = dup16(p2o[k] + so[k].mn);  // P2 <= 1744 and minPrev <= 2000: no u16 overflow
    p2x[k][1] = dup16(p2b[k] + sb[k].mn);
    m2[k][0] = dup16(so[k].mn);
    m2[k][1] = dup16(sb[k].mn);
  }
#pragma unroll
  for (int i = 0; i < NR; i++) {
#pragma unroll
    for (int k = 0; k < NC; k++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const V<LPT>& nb = h == 0 ? so[k].L : sb[k].L;
        const uint32_t lm = pair_of(i == 0 ? prev[k][h] : nb.r[i - 1], nb.r[i]);
        const uint32_t lp = pair_of(nb.r[i], i == NR - 1 ? next[k][h] : nb.r[i + 1]);
        uint32_t t = vmin2(lm, lp) + p1x2;
        t = vmin2(vmin2(t, nb.r[i]), p2x[k][h]);
        uint32_t lc = t + raw2[k].r[i] - m2[k][h];
        if (!FULL) lc = active ? lc : kInit2;
        if (h == 0) outo[k].r[i] = lc;
        else outb[k].r[i] = lc;
        rm[k][h] = vmin2(rm[k][h], lc);
        acc[k].r[i] += lc;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < NC; k++) {
    mino[k] = warp_min<LPT>(rm[k][0]);
    minb[k] = warp_min<LPT>(rm[k][1]);
  }
}

// The pixel of chain j at step s, in pass coordinates.
LUX_DEV void chain_pixel(const SplitArgs& a, int j, int s, int& xm, int& ym) {
  if (a.group == 0) {
    xm = s;
    ym = j;
  } else {
    xm = a.u.W - 1 - j;
    ym = s;
  }
}
LUX_DEV size_t pixel_index(const UniArgs& u, int xm, int ym, bool pass2) {  // memory index of a pass pixel
  const int x = pass2 ? u.W - 1 - xm : xm, y = pass2 ? u.H - 1 - ym : ym;
  return (size_t)y * u.W + x;
}

// The neighbour-path state that chain 0 of the block with index cb reads at step s + 1 (chain -1 at step s).
template <int LPT, bool PASS2>
LUX_DEV void chain_above(const SplitArgs& a, const uint16_t* bnd_up, const uint16_t* bnd_up_min, int cb, int s, Src<LPT>& u,
                         int lane) {
  constexpr int Dp = Dp_of(LPT);
  if (cb > 0) {
    vload<LPT>(u.L, bnd_up + (size_t)s * Dp, lane);
    u.mn = __ldcg(bnd_up_min + s);
  } else if (PASS2 && a.group == 0) {  // row -1 of pass -1: pass +1's final row y_b, path 1
    src_edge<LPT>(a.u, u, a.u.W - 1 - s, 1, lane);
  } else {  // row -1 of pass +1 (never written) or column W (the margin)
    src_init(u);
  }
}

// Bytes of one chain's staging slot of a step: [agg 2n B when read][raw n B], rounded up to 16 bytes (the kernel's layout
// and the launch's shared-memory size both come from here).
__host__ __device__ constexpr int chain_slot_bytes(int n, bool read_agg) { return ((read_agg ? 2 * n : 0) + n + 15) & ~15; }

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

// The hand-over between blocks: the block's last chain writes each step's L vector and minimum into its band buffer with
// bit 15 of every u16 set (L and its minimum stay below 2001, so the bit is free), and the next block's loader polls the
// entries themselves until every u16 of the step carries the bit. The buffer is cleared before each launch and each entry
// is written once per launch, so a set bit can only mean this launch's value; no fence or progress counter sits between
// the two blocks. Relaxed GPU-scope accesses of a lane's planes (16, 8 or 4 bytes) and of one u16.
constexpr uint32_t kMark2 = 0x80008000u;
template <int LPT>
LUX_DEV void st_marked(uint16_t* p, const V<LPT>& v, int lane) {
  uint32_t* q = reinterpret_cast<uint32_t*>(p + lane * LPT);
  if constexpr (LPT == 8)
    asm volatile("st.relaxed.gpu.global.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(q), "r"(v.r[0] | kMark2), "r"(v.r[1] | kMark2),
                 "r"(v.r[2] | kMark2), "r"(v.r[3] | kMark2) : "memory");
  else if constexpr (LPT == 4)
    asm volatile("st.relaxed.gpu.global.v2.u32 [%0], {%1, %2};" ::"l"(q), "r"(v.r[0] | kMark2), "r"(v.r[1] | kMark2) : "memory");
  else
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(q), "r"(v.r[0] | kMark2) : "memory");
}
// Loads a marked entry; returns whether every u16 of it carries the mark, and the values without it.
template <int LPT>
LUX_DEV bool ld_marked(const uint16_t* p, V<LPT>& v, int lane) {
  const uint32_t* q = reinterpret_cast<const uint32_t*>(p + lane * LPT);
  if constexpr (LPT == 8)
    asm volatile("ld.relaxed.gpu.global.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.r[0]), "=r"(v.r[1]), "=r"(v.r[2]), "=r"(v.r[3]) : "l"(q) : "memory");
  else if constexpr (LPT == 4)
    asm volatile("ld.relaxed.gpu.global.v2.u32 {%0, %1}, [%2];" : "=r"(v.r[0]), "=r"(v.r[1]) : "l"(q) : "memory");
  else
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v.r[0]) : "l"(q) : "memory");
  uint32_t all = kMark2;
#pragma unroll
  for (int i = 0; i < LPT / 2; i++) {
    all &= v.r[i];
    v.r[i] &= ~kMark2;
  }
  return all == kMark2;
}
LUX_DEV void st_marked16(uint16_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u16 [%0], %1;" ::"l"(p), "h"((unsigned short)(v | 0x8000u)) : "memory");
}
LUX_DEV bool ld_marked16(const uint16_t* p, uint32_t& v) {
  unsigned short t;
  asm volatile("ld.relaxed.gpu.global.u16 %0, [%1];" : "=h"(t) : "l"(p) : "memory");
  v = t & 0x7fffu;
  return (t & 0x8000u) != 0;
}

// One path step of a lane's planes (DenseStereoSgm.cs:276-313) with the neighbour's minimum carried in both u16 halves:
// the d-1 / d+1 words come from one byte permute per pair (the pair of planes 2i+1, 2i+2 is the d+1 word of pair i and
// the d-1 word of pair i+1). p2d: this path's P2 in both halves. Returns the new L and its warp minimum (both halves).
template <int LPT, bool FULL>
LUX_DEV void lean_path(const V<LPT>& nb, uint32_t md, uint32_t p2d, uint32_t p1x2, const V<LPT>& raw2, bool active, int lane,
                       V<LPT>& out, uint32_t& mdo) {
  constexpr int NR = LPT / 2;
  uint32_t prev = __shfl_up_sync(0xffffffffu, nb.r[NR - 1], 1);
  uint32_t next = __shfl_down_sync(0xffffffffu, nb.r[0], 1);
  if (lane == 0) prev = kInit2;   // plane -1: 2000
  if (lane == 31) next = kInit2;  // plane n (or a padding lane): 2000
  const uint32_t p2x = p2d + md;  // P2 + minPrev <= 3744 in each half: no carry between the halves
  uint32_t u[NR + 1];
  u[0] = pair_of(prev, nb.r[0]);
#pragma unroll
  for (int i = 0; i + 1 < NR; i++) u[i + 1] = pair_of(nb.r[i], nb.r[i + 1]);
  u[NR] = pair_of(nb.r[NR - 1], next);
  uint32_t m = 0xffffffffu;
#pragma unroll
  for (int i = 0; i < NR; i++) {
    uint32_t t = vmin2(u[i], u[i + 1]) + p1x2;  // min(L[d-1], L[d+1]) + P1
    t = vmin2(vmin2(t, nb.r[i]), p2x);          // with L[d] and P2 + minPrev
    uint32_t lc = t + raw2.r[i] - md;            // raw + m - minPrev, each half in [0, 2000)
    if (!FULL) lc = active ? lc : kInit2;        // padding lanes keep 2000
    out.r[i] = lc;
    m = vmin2(m, lc);
  }
  m = vmin2(m, __byte_perm(m, 0, 0x1032));
  mdo = __reduce_min_sync(0xffffffffu, m);
}

// The path groups of one pass. Chains of the block: two per chain warp (A from the warp above through the ring, B from
// A's previous step in registers); warp nw is the loader (chain j0-1 from the block above's band buffer into ring nw),
// warp nw+1 the publisher (the block's last chain out to its band buffer). A step's raw costs, aggregates and P2 are read
// straight from HBM two steps ahead into registers; the ring hands over one L vector and its minimum (both halves) per
// step through shared memory, ordered by full / empty mbarriers.
template <int LPT, bool FULL, bool PASS2, int GROUP>
__global__ void __launch_bounds__(kMaxWarpsS * 32, 1) k_chains(const SplitArgs a) {
  constexpr int NR = LPT / 2, Dp = Dp_of(LPT), kBatch = 4;
  const UniArgs& u = a.u;
  const int nw = (int)(blockDim.x >> 5) - 2;  // chain warps of this launch (two chains each)
  extern __shared__ __align__(16) uint16_t smem_chain[];
  auto ring = [&](int set, int slot) { return smem_chain + ((size_t)set * kRingS + slot) * Dp; };
  uint32_t* ring_md = reinterpret_cast<uint32_t*>(smem_chain + (size_t)(kMaxChainWarps + 1) * kRingS * Dp);
  auto rmd = [&](int set, int slot) -> uint32_t& { return ring_md[set * kRingS + slot]; };
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring_md + (kMaxChainWarps + 1) * kRingS);
  auto full = [&](int set, int slot) { return bars + set * kRingS + slot; };
  auto empty = [&](int set, int slot) { return bars + (kMaxChainWarps + 1) * kRingS + set * kRingS + slot; };
  // staging: per chain warp kStageS slots of [chain][agg 2n B (when read), raw n B]
  uint8_t* stage_base = reinterpret_cast<uint8_t*>(bars + 2 * (kMaxChainWarps + 1) * kRingS);
  __shared__ int s_cb;
  __shared__ volatile int s_stop;
  __shared__ float s_planes[256];  // the WTA's plane depths (group B of pass -1)
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (GROUP == 1 && PASS2)
    for (int i = tid; i < u.n; i += blockDim.x) s_planes[i] = u.planes[i];
  if (tid == 0) {
    s_cb = atomicAdd(u.ticket, 1);
    s_stop = 0;
  }
  for (int i = tid; i < 2 * (kMaxChainWarps + 1) * kRingS; i += blockDim.x) mbar_init(bars + i, 1);  // blocks may be small
  __syncthreads();
  const int cb = s_cb;
  const int j0 = cb * 2 * nw;
  const bool below_exists = j0 + 2 * nw < a.nchains;  // a block after this one reads its last chain
  const bool active = FULL || lane * LPT < u.n;
  const uint16_t* bnd_up = a.bnd + (size_t)(cb > 0 ? cb - 1 : 0) * a.nsteps * Dp;
  const uint16_t* bnd_up_min = a.bnd_min + (size_t)(cb > 0 ? cb - 1 : 0) * a.nsteps;
  uint16_t* bnd_me = a.bnd + (size_t)cb * a.nsteps * Dp;
  uint16_t* bnd_me_min = a.bnd_min + (size_t)cb * a.nsteps;
  // slot s & (kRingS - 1) of a ring holds step s; waits are bounded (a timeout stops the block with error 11)
  auto wait_filled = [&](int set, int s) {
    return mbar_wait(full(set, s & (kRingS - 1)), (uint32_t)(s / kRingS) & 1u, &s_stop, u.err, u.timeout_ns);
  };
  auto wait_free = [&](int set, int s) {
    return s < kRingS || mbar_wait(empty(set, s & (kRingS - 1)), (uint32_t)(s / kRingS - 1) & 1u, &s_stop, u.err, u.timeout_ns);
  };

  if (w == nw) {
    // ---------------- loader: chain j0-1 into ring nw ----------------
    // (group B's first block has none: its chain 0 is column c, whose path-3 neighbour is the margin)
    if (j0 < a.nchains && !(GROUP == 1 && cb == 0)) {
      const bool stalled = cb == u.stall_block;  // failure-path tests: this block's upstream entries never count as written
      const uint64_t t0 = global_ns();
      for (int sb = 0; sb < a.nsteps && !s_stop; sb += kBatch) {
        const int se = min(a.nsteps, sb + kBatch);
        bool ok = true;
        for (int s = sb; s < se && ok; s++) ok = wait_free(nw, s);
        if (!ok) break;
        Src<LPT> st[kBatch];
        if (cb > 0) {
          // poll the band buffer entries of steps sb..se-1 of the block above until all of them are written
          for (unsigned it = 0;; it++) {
            bool ready = !stalled;
#pragma unroll
            for (int k = 0; k < kBatch; k++) {
              if (sb + k >= se) break;
              ready &= ld_marked<LPT>(bnd_up + (size_t)(sb + k) * Dp, st[k].L, lane);
              uint32_t mn = 0;
              const bool mk = ld_marked16(bnd_up_min + sb + k, mn);
              st[k].mn = mn;
              ready &= mk;
            }
            if (__all_sync(0xffffffffu, ready)) break;
            __nanosleep(64);
            if ((it & 15) == 15 && (s_stop || *(volatile int*)u.err != 0 || global_ns() - t0 > u.timeout_ns)) {
              if (lane == 0) {
                atomicCAS(u.err, 0, 11);
                s_stop = 1;
              }
              ok = false;
              break;
            }
          }
          if (!ok) break;
        } else {
#pragma unroll
          for (int k = 0; k < kBatch; k++)
            if (sb + k < se) chain_above<LPT, PASS2>(a, bnd_up, bnd_up_min, cb, sb + k, st[k], lane);
        }
#pragma unroll
        for (int k = 0; k < kBatch; k++) {
          if (sb + k >= se) break;
          const int sl = (sb + k) & (kRingS - 1);
          sstore<LPT>(st[k].L, ring(nw, sl), lane);
          if (lane == 0) rmd(nw, sl) = dup16(st[k].mn);
        }
        __syncwarp();
        if (lane == 0)
          for (int s = sb; s < se; s++) mbar_arrive(full(nw, s & (kRingS - 1)));
      }
    }
    return;
  }
  if (w == nw + 1) {
    // ---------------- publisher: the block's last chain into its global band buffer ----------------
    if (below_exists) {
      for (int s = 0; s < a.nsteps; s++) {
        if (!wait_filled(nw - 1, s)) break;
        const int sl = s & (kRingS - 1);
        V<LPT> v;
        sload<LPT>(v, ring(nw - 1, sl), lane);
        st_marked<LPT>(bnd_me + (size_t)s * Dp, v, lane);
        if (lane == 0) st_marked16(bnd_me_min + s, rmd(nw - 1, sl) & 0xffffu);
        __syncwarp();
        if (lane == 0) mbar_arrive(empty(nw - 1, sl));
      }
    }
    return;
  }

  // ---------------- two chains: jA takes its neighbour from the warp above, jB from jA's previous step ----------------
  const int jA = j0 + 2 * w;
  if (jA >= a.nchains) return;
  const bool hasB = jA + 1 < a.nchains;  // else chain B repeats chain A's pixels and stores nothing
  const int jB = hasB ? jA + 1 : jA;
  const int up_set = w == 0 ? nw : w - 1;
  const bool has_consumer = jA + 2 < a.nchains;  // chain jB + 1 reads this warp's ring
  const int c = u.W - 1;
  const bool colc = GROUP == 1 && jA == 0;  // the last column: revisits, the special path-2 read
  const uint32_t p1x2 = dup16((uint32_t)u.p1);
  const int n = u.n;
  // consecutive steps of a chain are dpix pixels apart in memory, its P2 table entries dp2 apart
  const int dpix = GROUP == 0 ? (PASS2 ? -1 : 1) : (PASS2 ? -u.W : u.W);
  const int dp2 = GROUP == 0 ? 1 : u.W;
  constexpr bool kReadAgg = PASS2 || GROUP == 1;  // A of pass +1 is the first writer
  // per chain: memory pixel index and P2 index of the current step, own-path state (path 0 / 2) and its minimum
  int pix[2], p2i[2];
  V<LPT> oL[2];
  uint32_t om[2];
  const int jj[2] = {jA, jB};
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const int xm0 = GROUP == 0 ? 0 : u.W - 1 - jj[k], ym0 = GROUP == 0 ? jj[k] : 0;
    pix[k] = (int)pixel_index(u, xm0, ym0, PASS2);
    p2i[k] = ym0 * u.W + xm0;
    Src<LPT> s0;
    if (GROUP == 1 && PASS2) src_edge<LPT>(u, s0, u.W - 1 - xm0, 2, lane);  // row -1 of pass -1: path 2 of row y_b
    else src_init(s0);
    oL[k] = s0.L;
    om[k] = dup16(s0.mn);
  }
  const uint32_t* p2w = reinterpret_cast<const uint32_t*>(u.p2t) + (GROUP == 0 ? 0 : 1);  // the P2 word of this group's paths
  struct In {
    RawB<LPT> raw;
    V<LPT> agg;
    uint32_t p2;
  };
  // Raw costs and aggregates are staged kStageS steps ahead by cp.async into this warp's slots: per step and chain
  // [agg 2n B (when read)][raw n B]; lane j < n/8 copies planes 8j..8j+7 (16 B of aggregates, 8 B of raw costs), and
  // each lane then reads its own LPT planes. One commit group per step (empty past the chain's end).
  const int cbytes = chain_slot_bytes(n, kReadAgg);  // one chain's bytes of a step
  const int gran = n >> 3;
  uint8_t* stage = stage_base + (size_t)w * kStageS * 2 * cbytes;
  auto stage_at = [&](int slot, int k) { return stage + ((size_t)slot * 2 + k) * cbytes; };
  auto issue = [&](int s) {
    if (s < a.nsteps && lane < gran) {
#pragma unroll
      for (int k = 0; k < 2; k++) {
        if (k == 1 && !hasB) break;
        const long long pi = (long long)pix[k] + (long long)dpix * s;
        uint8_t* d = stage_at(s % kStageS, k);
        if constexpr (kReadAgg) cp_async16(d + lane * 16, reinterpret_cast<const uint8_t*>(u.agg + pi * n) + lane * 16);
        cp_async8(d + (kReadAgg ? 2 * n : 0) + lane * 8, u.raw + pi * n + lane * 8);
      }
    }
    cp_async_commit();
  };
  auto staged = [&](int k, int s, In& q) {  // chain k's inputs of step s from its slot (after the step's group completed)
    const uint8_t* d = stage_at(s % kStageS, hasB ? k : 0);
    if (!active) {
      q.raw.r[0] = 0;
      if constexpr (LPT >= 8) q.raw.r[1] = 0;
#pragma unroll
      for (int i = 0; i < NR; i++) q.agg.r[i] = 0;
      return;
    }
    const uint8_t* r = d + (kReadAgg ? 2 * n : 0) + lane * LPT;
    if constexpr (LPT == 8) {
      const uint2 t = *reinterpret_cast<const uint2*>(r);
      q.raw.r[0] = t.x;
      q.raw.r[1] = t.y;
    } else if constexpr (LPT == 4) {
      q.raw.r[0] = *reinterpret_cast<const uint32_t*>(r);
    } else {
      q.raw.r[0] = *reinterpret_cast<const uint16_t*>(r);
    }
    if constexpr (kReadAgg) {
      V<LPT> v;
      sload<LPT>(v, reinterpret_cast<const uint16_t*>(d), lane);
      q.agg = v;
    }
  };
  auto fetch = [&](int k, int s, In& q) { q.p2 = __ldg(p2w + 2 * (long long)(p2i[k] + dp2 * s)); };  // step s's P2 word
  // revisit R(c, y) of paths 2 and 3 (column c only): adds them to agg(c, y), keeps R.p2 for later revisits
  auto revisit23 = [&](int y) {
    Src<LPT> s2[1], s3[1];
    const int e = u.src2[y], kind = src_kind(e), row = src_row(e);
    if (kind == kSrcInit) src_init(s2[0]);
    else if (kind == kSrcEdge) src_edge<LPT>(u, s2[0], PASS2 ? 0 : c, 2, lane);
    else src_cs<LPT>(u, s2[0], row, kind - kSrcCs, c, lane);
    src_init(s3[0]);
    const float4 g = pix_of(u, c, y);
    int p2 = 0;
    if (lane < 2) p2 = p2_of(u, g, lane == 0 ? s2[0].pix : s3[0].pix);
    const uint32_t P2a[1] = {(uint32_t)__shfl_sync(0xffffffffu, p2, 0)}, P2b[1] = {(uint32_t)__shfl_sync(0xffffffffu, p2, 1)};
    const size_t pi = pixel_index(u, c, y, PASS2);
    V<LPT> raw2[1], acc[1], o2[1], o3[1];
    load_raw<LPT>(u, c, y, raw2[0], active, lane);
    uint16_t* ap = u.agg + pi * u.n + lane * LPT;
    agg_load<LPT>(ap, acc[0], active);
    uint32_t m2[1], m3[1];
    chain_paths<LPT, FULL, 1>(s2, P2a, s3, P2b, p1x2, raw2, active, lane, o2, o3, acc, m2, m3);
    agg_store<LPT>(ap, acc[0], active);
    cs_put<LPT>(u, o2[0], m2[0], y, 4, lane);
    if (!PASS2 && (u.extra[y] & 1)) {  // R(y_b) is what pass -1 will read at the last column
      vstore<LPT>(o2[0], u.edge + ((size_t)c * 3 + 1) * Dp, lane);
      if (lane == 0) __stcg(u.edge_min + (size_t)c * 3 + 1, (uint16_t)m2[0]);
    }
    __syncwarp();
  };
  V<LPT> pbL;  // chain A's neighbour-path output of the previous step: chain B's neighbour
  uint32_t pbm = kInit2;
  vinit(pbL);
  auto step = [&](int s, In (&q)[2]) -> bool {
    // ---- hand-over in: the warp above finished step s-1; the warp below is done with the slot this step reuses ----
    const bool nb_ring = s > 0 && !colc;
    if (nb_ring && !wait_filled(up_set, s - 1)) return false;
    if (has_consumer && !wait_free(w, s)) return false;
    int xm[2], ym[2];
    chain_pixel(a, jA, s, xm[0], ym[0]);
    chain_pixel(a, jB, s, xm[1], ym[1]);
    if (colc) {  // revisits that the reference runs before N(c, y), and the special path-2 read
      const int cnt = u.batch_count[ym[0]], fr = u.batch_first[ym[0]];
      for (int k = 0; k < cnt; k++) revisit23(fr + k);
      if (u.flags[ym[0]] & 1) {
        Src<LPT> r;
        src_cs<LPT>(u, r, ym[0] - 1, 4, c, lane);
        oL[0] = r.L;
        om[0] = dup16(r.mn);
      }
    }
    V<LPT> nbL[2];
    uint32_t nbm[2];
    if (nb_ring) {
      const int sl = (s - 1) & (kRingS - 1);
      sload<LPT>(nbL[0], ring(up_set, sl), lane);
      nbm[0] = rmd(up_set, sl);
    } else if (GROUP == 1 && PASS2 && !colc) {  // row -1 of pass -1: path 3 of pass +1's row y_b at x+1
      Src<LPT> e;
      src_edge<LPT>(u, e, u.W - 1 - (xm[0] + 1), 3, lane);
      nbL[0] = e.L;
      nbm[0] = dup16(e.mn);
    } else {
      vinit(nbL[0]);
      nbm[0] = kInit2;
    }
    if (s > 0) {
      nbL[1] = pbL;
      nbm[1] = pbm;
    } else if (GROUP == 1 && PASS2) {
      Src<LPT> e;
      src_edge<LPT>(u, e, u.W - 1 - (xm[1] + 1), 3, lane);
      nbL[1] = e.L;
      nbm[1] = dup16(e.mn);
    } else {
      vinit(nbL[1]);
      nbm[1] = kInit2;
    }
    cp_async_wait<kStageS - 1>();  // this lane's copies of step s have landed
    __syncwarp();                  // and every lane's
    staged(0, s, q[0]);
    staged(1, s, q[1]);
    __syncwarp();  // every lane has read the slot before it is refilled
    issue(s + kStageS);
    V<LPT> oo[2], ob[2], acc[2];
    uint32_t mo[2], mb[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
      V<LPT> raw2;
      raw_unpack<LPT>(q[k].raw, raw2);
      lean_path<LPT, FULL>(oL[k], om[k], dup16(q[k].p2 & 0xffffu), p1x2, raw2, active, lane, oo[k], mo[k]);
      lean_path<LPT, FULL>(nbL[k], nbm[k], __byte_perm(q[k].p2, 0, 0x3232), p1x2, raw2, active, lane, ob[k], mb[k]);
#pragma unroll
      for (int i = 0; i < NR; i++) acc[k].r[i] = (kReadAgg ? q[k].agg.r[i] : 0u) + oo[k].r[i] + ob[k].r[i];
    }
    // ---- hand-over out: chain B's neighbour-path state for the warp below ----
    const int sl = s & (kRingS - 1);
    if (has_consumer) {
      sstore<LPT>(ob[1], ring(w, sl), lane);
      if (lane == 0) rmd(w, sl) = mb[1];
    }
    __syncwarp();
    if (lane == 0) {
      if (has_consumer) mbar_arrive(full(w, sl));
      if (nb_ring) mbar_arrive(empty(up_set, (s - 1) & (kRingS - 1)));
    }
    // ---- aggregates, WTA, the states kept for revisits and for pass -1 ----
#pragma unroll
    for (int k = 0; k < 2; k++) {
      if (k == 1 && !hasB) break;
      const size_t pi = (size_t)(pix[k] + dpix * s);
      uint16_t* ap = u.agg + pi * n + lane * LPT;
      if (GROUP == 1 && PASS2 && !(k == 0 && colc)) {
        if (u.keep_agg) agg_store<LPT>(ap, acc[k], active);
        const int arg = wta_arg<LPT>(acc[k], active, lane);
        if (lane == 0) u.depth[pi] = s_planes[arg];
      } else {
        agg_store<LPT>(ap, acc[k], active);
      }
      if (GROUP == 0 && xm[k] == c - 1) {  // N(c-1): paths 0 and 1 are revisit sources
        cs_put<LPT>(u, oo[k], mo[k] & 0xffffu, ym[k], 0, lane);
        cs_put<LPT>(u, ob[k], mb[k] & 0xffffu, ym[k], 1, lane);
      }
      if (k == 0 && colc) cs_put<LPT>(u, oo[0], mo[0] & 0xffffu, ym[0], 2, lane);  // N(c).p2
      if (!PASS2 && ym[k] == u.y_b) {  // pass +1's row y_b: what pass -1 reads above its first row
        if (GROUP == 0) {
          vstore<LPT>(ob[k], u.edge + ((size_t)xm[k] * 3 + 0) * Dp, lane);
          if (lane == 0) __stcg(u.edge_min + (size_t)xm[k] * 3 + 0, (uint16_t)(mb[k] & 0xffffu));
        } else {
          vstore<LPT>(oo[k], u.edge + ((size_t)xm[k] * 3 + 1) * Dp, lane);
          vstore<LPT>(ob[k], u.edge + ((size_t)xm[k] * 3 + 2) * Dp, lane);
          if (lane == 0) {
            __stcg(u.edge_min + (size_t)xm[k] * 3 + 1, (uint16_t)(mo[k] & 0xffffu));
            __stcg(u.edge_min + (size_t)xm[k] * 3 + 2, (uint16_t)(mb[k] & 0xffffu));
          }
        }
      }
    }
    oL[0] = oo[0];
    om[0] = mo[0];
    oL[1] = oo[1];
    om[1] = mo[1];
    pbL = ob[0];
    pbm = mb[0];
    return true;
  };
  // Step s reads queue entry s & 1: the inputs of step s + 2 are fetched once step s has consumed its entry.
  for (int s = 0; s < kStageS; s++) issue(s);
  In q0[2], q1[2];
  fetch(0, 0, q0[0]);
  fetch(1, 0, q0[1]);
  if (a.nsteps > 1) {
    fetch(0, 1, q1[0]);
    fetch(1, 1, q1[1]);
  }
  bool ok = true;
  for (int s = 0; s < a.nsteps; s += 2) {
    if (!step(s, q0)) {
      ok = false;
      break;
    }
    if (s + 2 < a.nsteps) {
      fetch(0, s + 2, q0[0]);
      fetch(1, s + 2, q0[1]);
    }
    if (s + 1 >= a.nsteps) break;
    if (!step(s + 1, q1)) {
      ok = false;
      break;
    }
    if (s + 3 < a.nsteps) {
      fetch(0, s + 3, q1[0]);
      fetch(1, s + 3, q1[1]);
    }
  }
  cp_async_wait<0>();  // no copy is in flight when the warp leaves
  if (ok && colc)  // the last band's revisits when no later visit of the column follows them
    for (int k = 0; k < u.end_count; k++) revisit23(u.end_first + k);
}

// Paths 0 and 1 of the revisits R(c, y) (column c-1 states or the boundary): one warp per revisit row.
template <int LPT, bool FULL, bool PASS2>
__global__ void k_revisit01(const SplitArgs a) {
  const UniArgs& u = a.u;
  const int lane = threadIdx.x & 31;
  const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (k >= a.n_rev) return;
  const int y = a.rev_rows[k];
  const int c = u.W - 1;
  const bool active = FULL || lane * LPT < u.n;
  Src<LPT> s0[1], s1[1];
  const int e0 = u.src0[y], e1 = u.src1[y];
  if (src_kind(e0) == kSrcInit) src_init(s0[0]);
  else src_cs<LPT>(u, s0[0], src_row(e0), src_kind(e0) - kSrcCs, c - 1, lane);
  if (src_kind(e1) == kSrcInit) src_init(s1[0]);
  else if (src_kind(e1) == kSrcEdge) src_edge<LPT>(u, s1[0], PASS2 ? 1 : c - 1, 1, lane);
  else src_cs<LPT>(u, s1[0], src_row(e1), src_kind(e1) - kSrcCs, c - 1, lane);
  const float4 g = pix_of(u, c, y);
  int p2 = 0;
  if (lane < 2) p2 = p2_of(u, g, lane == 0 ? s0[0].pix : s1[0].pix);
  const uint32_t P2a[1] = {(uint32_t)__shfl_sync(0xffffffffu, p2, 0)}, P2b[1] = {(uint32_t)__shfl_sync(0xffffffffu, p2, 1)};
  const size_t pi = pixel_index(u, c, y, PASS2);
  V<LPT> raw2[1], acc[1], o0[1], o1[1];
  load_raw<LPT>(u, c, y, raw2[0], active, lane);
  uint16_t* ap = u.agg + pi * u.n + lane * LPT;
  agg_load<LPT>(ap, acc[0], active);
  const uint32_t p1x2 = dup16((uint32_t)u.p1);
  uint32_t m0[1], m1[1];
  chain_paths<LPT, FULL, 1>(s0, P2a, s1, P2b, p1x2, raw2, active, lane, o0, o1, acc, m0, m1);
  agg_store<LPT>(ap, acc[0], active);
  if (!PASS2 && (u.extra[y] & 1)) {  // R(y_b) is what pass -1 will read at the last column
    constexpr int D = Dp_of(LPT);
    vstore<LPT>(o1[0], u.edge + ((size_t)c * 3 + 0) * D, lane);
    if (lane == 0) __stcg(u.edge_min + (size_t)c * 3 + 0, (uint16_t)m1[0]);
  }
}

// Chain warps per block: enough that every chain of the launch is resident at once (one block per SM), within the
// register file; and the block count that follows.
int g_sm_count = 0;
int chain_warps(int nchains) {
  if (g_sm_count <= 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || g_sm_count <= 0) g_sm_count = 148;
  }
  const int warps = (nchains + 1) / 2;
  return std::max(1, std::min(kMaxChainWarps, (warps + g_sm_count - 1) / g_sm_count));
}
int chain_blocks(int nchains) {
  const int per = 2 * chain_warps(nchains);
  return (nchains + per - 1) / per;
}

// Dynamic shared memory of a launch: the rings, their minima (u32 each) and their full / empty mbarriers.
template <int LPT>
size_t chain_smem_bytes(int nw, int n, bool read_agg) {
  const size_t rings = (size_t)(kMaxChainWarps + 1) * kRingS * Dp_of(LPT) * 2 + (size_t)(kMaxChainWarps + 1) * kRingS * 4 +
                       (size_t)2 * (kMaxChainWarps + 1) * kRingS * 8;
  const size_t staging = (size_t)nw * kStageS * 2 * (size_t)chain_slot_bytes(n, read_agg);
  return rings + staging;
}

template <int LPT, bool FULL, bool PASS2, int GROUP>
void launch_chains_t(const SplitArgs& a, cudaStream_t s) {
  const int nw = chain_warps(a.nchains);
  // every band-buffer entry this launch reads starts unwritten (bit 15 clear)
  const size_t entries = (size_t)chain_blocks(a.nchains) * a.nsteps;
  cudaMemsetAsync(a.bnd, 0, entries * Dp_of(LPT) * 2, s);
  cudaMemsetAsync(a.bnd_min, 0, entries * 2, s);
  const size_t smem = chain_smem_bytes<LPT>(nw, a.u.n, PASS2 || GROUP == 1);
  static size_t configured = 0;
  if (smem > configured) {
    cudaFuncSetAttribute(k_chains<LPT, FULL, PASS2, GROUP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    configured = smem;
  }
  k_chains<LPT, FULL, PASS2, GROUP><<<chain_blocks(a.nchains), (nw + 2) * 32, smem, s>>>(a);
  count_launches(1);
}

template <int LPT, bool FULL, bool PASS2>
void launch_pass_groups(SplitArgs& a, int* progA, int* progB, cudaStream_t s) {
  const UniArgs base = a.u;
  // group A: chains = rows
  a.group = 0;
  a.nchains = base.H;
  a.nsteps = base.W;
  a.u.progress = progA;
  a.u.ticket = progA + chain_blocks(base.H);
  launch_chains_t<LPT, FULL, PASS2, 0>(a, s);
  if (a.n_rev > 0) {
    k_revisit01<LPT, FULL, PASS2><<<(a.n_rev * 32 + 127) / 128, 128, 0, s>>>(a);
    count_launches(1);
  }
  // group B: chains = columns from the right
  a.group = 1;
  a.nchains = base.W;
  a.nsteps = base.H;
  a.u.progress = progB;
  a.u.ticket = progB + chain_blocks(base.W);
  launch_chains_t<LPT, FULL, PASS2, 1>(a, s);
  a.u = base;
}

template <int LPT>
void launch_pass_split(SplitArgs& a, int* progA, int* progB, bool pass2, cudaStream_t s) {
  const bool full = a.u.n == 32 * LPT;
  if (!pass2) {
    if (full) launch_pass_groups<LPT, true, false>(a, progA, progB, s);
    else launch_pass_groups<LPT, false, false>(a, progA, progB, s);
  } else {
    if (full) launch_pass_groups<LPT, true, true>(a, progA, progB, s);
    else launch_pass_groups<LPT, false, true>(a, progA, progB, s);
  }
}

int lpt_of(int n) { return n <= 64 ? 2 : n <= 128 ? 4 : 8; }

struct SplitLayout {
  size_t bnd, bnd_min, prog, edge, edge_min, cs, cs_min, sched, p2t, total;
};

SplitLayout split_layout(int W, int H, int n) {
  const size_t Dp = 32 * (size_t)lpt_of(n);
  const int nA = chain_blocks(H), nB = chain_blocks(W);
  const size_t L = std::max((size_t)nA * W, (size_t)nB * H);  // block buffers of group A, then reused by group B
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  SplitLayout s;
  size_t o = 0;
  s.bnd = o; o += al(L * Dp * 2);
  s.bnd_min = o; o += al(L * 2);
  s.prog = o; o += al((size_t)2 * (nA + 1 + nB + 1) * 4);  // per pass: A counters + ticket, B counters + ticket
  s.edge = o; o += al((size_t)W * 3 * Dp * 2);
  s.edge_min = o; o += al((size_t)W * 3 * 2);
  s.cs = o; o += al((size_t)H * 5 * Dp * 2);
  s.cs_min = o; o += al((size_t)H * 5 * 2);
  s.sched = o; o += al((size_t)2 * 8 * H * 4);  // per pass: 7 schedule columns + the revisit row list
  s.p2t = o; o += al((size_t)W * H * 8);
  s.total = o;
  return s;
}

}  // namespace

size_t split_scratch_bytes(int W, int H, int n) { return split_layout(W, H, n).total; }

// k_p2_table and k_wta_column live in sgm_uniform.cu
void launch_p2_table(const UniArgs& a, uint2* p2t, cudaStream_t s);
void launch_wta_column(const uint16_t* agg, int W, int H, int n, const float* planes, float* depth, cudaStream_t s);

int run_sgm_split(const LayerGeom& g, int xsw, uint16_t p1, float p2scale, const float gw[4], const uint8_t* raw, uint16_t* agg,
                  uint16_t* agg_pass1, float* depth, int keep_agg, void* scratch, size_t scratch_bytes, int* err, cudaStream_t s) {
  if (xsw) return 12;
  const int W = g.W, H = g.H, n = g.n_planes, T = g.tile;
  const SplitLayout L = split_layout(W, H, n);
  if (scratch_bytes < L.total) return 9;
  char* base = static_cast<char*>(scratch);
  RevisitSchedule sch[2];
  std::vector<int> host((size_t)2 * 8 * H, 0);
  int n_rev[2] = {0, 0};
  for (int pass = 0; pass < 2; pass++) {
    build_revisit_schedule(W, H, T, pass == 1, sch[pass]);
    int* h = host.data() + (size_t)pass * 8 * H;
    const std::vector<int>* cols[7] = {&sch[pass].flags, &sch[pass].batch_first, &sch[pass].batch_count, &sch[pass].src0,
                                       &sch[pass].src1, &sch[pass].src2, &sch[pass].extra};
    for (int k = 0; k < 7; k++) std::memcpy(h + (size_t)k * H, cols[k]->data(), (size_t)H * 4);
    int* rl = h + (size_t)7 * H;  // every row with a revisit (batches and the end batch)
    for (int y = 0; y < H; y++)
      for (int k = 0; k < sch[pass].batch_count[y]; k++) rl[n_rev[pass]++] = sch[pass].batch_first[y] + k;
    for (int k = 0; k < sch[pass].end_count; k++) rl[n_rev[pass]++] = sch[pass].end_first + k;
  }
  int* dsched = reinterpret_cast<int*>(base + L.sched);
  if (cudaMemcpyAsync(dsched, host.data(), host.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return 10;
  const int nA = chain_blocks(H), nB = chain_blocks(W);
  int* prog = reinterpret_cast<int*>(base + L.prog);
  cudaMemsetAsync(prog, 0, (size_t)2 * (nA + 1 + nB + 1) * 4, s);
  SplitArgs a;
  std::memset(&a, 0, sizeof a);
  UniArgs& u = a.u;
  u.W = W; u.H = H; u.n = n; u.T = T;
  u.raw = raw; u.agg = agg; u.depth = depth; u.planes = g.planes; u.guidance = g.guidance;
  u.p1 = p1;
  volatile float p1f = (float)p1;
  u.p2base = p1f * p2scale;
  for (int i = 0; i < 4; i++) u.gw[i] = gw[i];
  a.bnd = reinterpret_cast<uint16_t*>(base + L.bnd);
  a.bnd_min = reinterpret_cast<uint16_t*>(base + L.bnd_min);
  u.edge = reinterpret_cast<uint16_t*>(base + L.edge);
  u.edge_min = reinterpret_cast<uint16_t*>(base + L.edge_min);
  u.cs = reinterpret_cast<uint16_t*>(base + L.cs);
  u.cs_min = reinterpret_cast<uint16_t*>(base + L.cs_min);
  u.y_b = sch[0].y_b;
  u.err = err;
  u.timeout_ns = g.timeout_ns;
  u.stall_block = g.stall_block;
  u.never = g.never;
  u.keep_agg = keep_agg;
  u.p2t = reinterpret_cast<const uint2*>(base + L.p2t);
  const int lpt = lpt_of(n);
  for (int pass = 0; pass < 2; pass++) {
    const int* h = dsched + (size_t)pass * 8 * H;
    u.flags = h; u.batch_first = h + H; u.batch_count = h + 2 * H; u.src0 = h + 3 * H; u.src1 = h + 4 * H; u.src2 = h + 5 * H;
    u.extra = h + 6 * H;
    a.rev_rows = h + 7 * H;
    a.n_rev = n_rev[pass];
    u.end_first = sch[pass].end_first;
    u.end_count = sch[pass].end_count;
    u.dir = pass == 0 ? 1 : -1;
    u.edge_write = pass == 0;
    u.edge_read = pass == 1;
    u.wta = pass == 1;
    launch_p2_table(u, reinterpret_cast<uint2*>(base + L.p2t), s);
    int* progA = prog + (size_t)pass * (nA + 1 + nB + 1);
    int* progB = progA + nA + 1;
    if (lpt == 2) launch_pass_split<2>(a, progA, progB, pass == 1, s);
    else if (lpt == 4) launch_pass_split<4>(a, progA, progB, pass == 1, s);
    else launch_pass_split<8>(a, progA, progB, pass == 1, s);
    if (pass == 0 && agg_pass1) cudaMemcpyAsync(agg_pass1, agg, (size_t)W * H * n * 2, cudaMemcpyDeviceToDevice, s);
  }
  launch_wta_column(agg, W, H, n, g.planes, depth, s);
  return 0;
}

}  // namespace lux
