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
constexpr int kPublishS = 8;           // global progress released every kPublishS steps
constexpr int kStage = 4;              // steps of HBM input staged ahead per chain

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

template <int LPT, bool FULL, bool PASS2, int GROUP>
__global__ void __launch_bounds__(kMaxWarpsS * 32, 1) k_chains(const SplitArgs a) {
  constexpr int NR = LPT / 2, Dp = Dp_of(LPT), kBatch = 4;
  const UniArgs& u = a.u;
  const int nw = (int)(blockDim.x >> 5) - 2;  // chain warps of this launch (two chains each)
  extern __shared__ __align__(16) uint16_t smem_chain[];
  auto ring = [&](int set, int slot) { return smem_chain + ((size_t)set * kRingS + slot) * Dp; };
  uint16_t* ring_min = smem_chain + (size_t)(kMaxChainWarps + 1) * kRingS * Dp;
  auto rmin_at = [&](int set, int slot) -> uint16_t& { return ring_min[set * kRingS + slot]; };
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring_min + (size_t)(kMaxChainWarps + 1) * kRingS + 8);
  auto full = [&](int set, int slot) { return bars + set * kRingS + slot; };
  auto empty = [&](int set, int slot) { return bars + (kMaxChainWarps + 1) * kRingS + set * kRingS + slot; };
  uint8_t* stage_base = reinterpret_cast<uint8_t*>(bars + 2 * (kMaxChainWarps + 1) * kRingS);  // 16-B aligned
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
      int avail = cb > 0 ? 0 : a.nsteps;
      for (int sb = 0; sb < a.nsteps && !s_stop; sb += kBatch) {
        const int se = min(a.nsteps, sb + kBatch);
        bool ok = true;
        for (int s = sb; s < se && ok; s++) ok = wait_free(nw, s);
        if (!ok) break;
        if (avail < se) {
          int v = 0;
          if (lane == 0) v = wait_at_least_value(cb == u.stall_block ? u.never : u.progress + (cb - 1), se, u.err, 11, u.timeout_ns);
          v = __shfl_sync(0xffffffffu, v, 0);
          __syncwarp();
          if (v < 0) {
            s_stop = 1;
            break;
          }
          avail = v;
        }
        Src<LPT> st[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; k++)
          if (sb + k < se) chain_above<LPT, PASS2>(a, bnd_up, bnd_up_min, cb, sb + k, st[k], lane);
#pragma unroll
        for (int k = 0; k < kBatch; k++) {
          if (sb + k >= se) break;
          const int sl = (sb + k) & (kRingS - 1);
          vstore_s<LPT>(st[k].L, ring(nw, sl), lane);
          if (lane == 0) rmin_at(nw, sl) = (uint16_t)st[k].mn;
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
        vload_s<LPT>(v, ring(nw - 1, sl), lane);
        vstore<LPT>(v, bnd_me + (size_t)s * Dp, lane);
        if (lane == 0) __stcg(bnd_me_min + s, rmin_at(nw - 1, sl));
        __syncwarp();
        if (lane == 0) mbar_arrive(empty(nw - 1, sl));
        if ((s + 1) % kPublishS == 0) st_release(u.progress + cb, s + 1);
      }
    }
    __syncwarp();
    if (lane == 0) st_release(u.progress + cb, a.nsteps);
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
  // memory step between consecutive steps of a chain (pixels), and the P2 table step
  const long long dpix = GROUP == 0 ? (PASS2 ? -1 : 1) : (PASS2 ? -(long long)u.W : (long long)u.W);
  const long long dp2 = GROUP == 0 ? 1 : u.W;
  struct Chain {
    long long pix0;     // memory index of the chain's first pixel
    const uint2* p2p0;  // its P2 table entry
    Src<LPT> own;       // the chain's own-path state (path 0 / 2) after the previous step
  };
  Chain ch[2];
  const int jj[2] = {jA, jB};
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const int xm0 = GROUP == 0 ? 0 : u.W - 1 - jj[k], ym0 = GROUP == 0 ? jj[k] : 0;
    ch[k].pix0 = (long long)pixel_index(u, xm0, ym0, PASS2);
    ch[k].p2p0 = u.p2t + (size_t)ym0 * u.W + xm0;
    if (GROUP == 1 && PASS2) src_edge<LPT>(u, ch[k].own, u.W - 1 - xm0, 2, lane);  // row -1 of pass -1: path 2 of row y_b
    else src_init(ch[k].own);
  }
  // HBM inputs of a step, staged kStage steps ahead by cp.async: per chain and slot [agg 2n B][raw n B][P2 8 B] (agg only
  // where it is read). The first n/8 lanes copy 16 B of aggregates and 8 B of raw costs each, lane 0 the P2 word.
  constexpr bool kReadAgg = PASS2 || GROUP == 1;  // A of pass +1 is the first writer
  const int n = u.n, gran = n >> 3;
  const int raw_off = kReadAgg ? 2 * n : 0, p2_off = raw_off + n;
  const int sbytes = (p2_off + 8 + 15) & ~15;
  uint8_t* stage = stage_base + (size_t)(2 * w) * kStage * sbytes;
  auto stage_at = [&](int k, int s) { return stage + ((size_t)k * kStage + (s % kStage)) * sbytes; };
  auto issue = [&](int s) {
    if (s < a.nsteps) {
#pragma unroll
      for (int k = 0; k < 2; k++) {
        uint8_t* d = stage_at(k, s);
        const long long pix = ch[k].pix0 + dpix * s;
        if (lane < gran) {
          if constexpr (kReadAgg) cp_async16(d + lane * 16, reinterpret_cast<const uint8_t*>(u.agg + pix * n) + lane * 16);
          cp_async8(d + raw_off + lane * 8, u.raw + pix * n + lane * 8);
        }
        if (lane == 0) cp_async8(d + p2_off, ch[k].p2p0 + dp2 * s);
      }
    }
    cp_async_commit();  // one group per step, empty past the end
  };
  struct Queued {
    RawB<LPT> raw;
    V<LPT> agg;
    uint32_t p2;
  };
  auto staged = [&](int k, int s, Queued& q) {  // after the step's group completed and a __syncwarp
    const uint8_t* d = stage_at(k, s);
    if (!active) {
      q.raw.r[0] = 0;
      if constexpr (LPT >= 8) q.raw.r[1] = 0;
#pragma unroll
      for (int i = 0; i < NR; i++) q.agg.r[i] = 0;
    } else {
      if constexpr (LPT == 8) {
        const uint2 t = *reinterpret_cast<const uint2*>(d + raw_off + lane * 8);
        q.raw.r[0] = t.x;
        q.raw.r[1] = t.y;
      } else if constexpr (LPT == 4) {
        q.raw.r[0] = *reinterpret_cast<const uint32_t*>(d + raw_off + lane * 4);
      } else {
        q.raw.r[0] = *reinterpret_cast<const uint16_t*>(d + raw_off + lane * 2);
      }
      if constexpr (kReadAgg) {
        if constexpr (LPT == 8) {
          const uint4 t = *reinterpret_cast<const uint4*>(d + lane * 16);
          q.agg.r[0] = t.x; q.agg.r[1] = t.y; q.agg.r[2] = t.z; q.agg.r[3] = t.w;
        } else if constexpr (LPT == 4) {
          const uint2 t = *reinterpret_cast<const uint2*>(d + lane * 8);
          q.agg.r[0] = t.x; q.agg.r[1] = t.y;
        } else {
          q.agg.r[0] = *reinterpret_cast<const uint32_t*>(d + lane * 4);
        }
      }
    }
    const uint2 pp = *reinterpret_cast<const uint2*>(d + p2_off);
    q.p2 = GROUP == 0 ? pp.x : pp.y;
  };
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
  Src<LPT> prevAb;  // chain A's neighbour-path output of the previous step: chain B's neighbour
  auto step = [&](int s) -> bool {
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
      if (u.flags[ym[0]] & 1) src_cs<LPT>(u, ch[0].own, ym[0] - 1, 4, c, lane);
    }
    Src<LPT> own[2] = {ch[0].own, ch[1].own}, nb[2];
    if (nb_ring) {
      const int sl = (s - 1) & (kRingS - 1);
      vload_s<LPT>(nb[0].L, ring(up_set, sl), lane);
      nb[0].mn = rmin_at(up_set, sl);
    } else if (GROUP == 1 && PASS2 && !colc) {  // row -1 of pass -1: path 3 of pass +1's row y_b at x+1
      src_edge<LPT>(u, nb[0], u.W - 1 - (xm[0] + 1), 3, lane);
    } else {
      src_init(nb[0]);
    }
    if (s > 0) nb[1] = prevAb;
    else if (GROUP == 1 && PASS2) src_edge<LPT>(u, nb[1], u.W - 1 - (xm[1] + 1), 3, lane);
    else src_init(nb[1]);
    Queued qa, qb;
    staged(0, s, qa);
    staged(1, s, qb);
    const uint32_t p2o[2] = {qa.p2 & 0xffffu, qb.p2 & 0xffffu}, p2b[2] = {qa.p2 >> 16, qb.p2 >> 16};
    V<LPT> raw2[2], acc[2], oo[2], ob[2];
    raw_unpack<LPT>(qa.raw, raw2[0]);
    raw_unpack<LPT>(qb.raw, raw2[1]);
    if constexpr (kReadAgg) {
      acc[0] = qa.agg;
      acc[1] = qb.agg;
    } else {
#pragma unroll
      for (int i = 0; i < NR; i++) acc[0].r[i] = acc[1].r[i] = 0;
    }
    uint32_t mo[2], mb[2];
    chain_paths<LPT, FULL, 2>(own, p2o, nb, p2b, p1x2, raw2, active, lane, oo, ob, acc, mo, mb);
    // ---- hand-over out: chain B's neighbour-path state for the warp below ----
    const int sl = s & (kRingS - 1);
    if (has_consumer) {
      vstore_s<LPT>(ob[1], ring(w, sl), lane);
      if (lane == 0) rmin_at(w, sl) = (uint16_t)mb[1];
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
      const size_t pi = pixel_index(u, xm[k], ym[k], PASS2);
      uint16_t* ap = u.agg + pi * u.n + lane * LPT;
      if (GROUP == 1 && PASS2 && !(k == 0 && colc)) {
        if (u.keep_agg) agg_store<LPT>(ap, acc[k], active);
        const int arg = wta_arg<LPT>(acc[k], active, lane);
        if (lane == 0) u.depth[pi] = s_planes[arg];
      } else {
        agg_store<LPT>(ap, acc[k], active);
      }
      if (GROUP == 0 && xm[k] == c - 1) {  // N(c-1): paths 0 and 1 are revisit sources
        cs_put<LPT>(u, oo[k], mo[k], ym[k], 0, lane);
        cs_put<LPT>(u, ob[k], mb[k], ym[k], 1, lane);
      }
      if (k == 0 && colc) cs_put<LPT>(u, oo[0], mo[0], ym[0], 2, lane);  // N(c).p2
      if (!PASS2 && ym[k] == u.y_b) {  // pass +1's row y_b: what pass -1 reads above its first row
        if (GROUP == 0) {
          vstore<LPT>(ob[k], u.edge + ((size_t)xm[k] * 3 + 0) * Dp, lane);
          if (lane == 0) __stcg(u.edge_min + (size_t)xm[k] * 3 + 0, (uint16_t)mb[k]);
        } else {
          vstore<LPT>(oo[k], u.edge + ((size_t)xm[k] * 3 + 1) * Dp, lane);
          vstore<LPT>(ob[k], u.edge + ((size_t)xm[k] * 3 + 2) * Dp, lane);
          if (lane == 0) {
            __stcg(u.edge_min + (size_t)xm[k] * 3 + 1, (uint16_t)mo[k]);
            __stcg(u.edge_min + (size_t)xm[k] * 3 + 2, (uint16_t)mb[k]);
          }
        }
      }
    }
    ch[0].own.L = oo[0];
    ch[0].own.mn = mo[0];
    ch[1].own.L = oo[1];
    ch[1].own.mn = mo[1];
    prevAb.L = ob[0];
    prevAb.mn = mb[0];
    return true;
  };
  for (int s = 0; s < kStage; s++) issue(s);
  bool ok = true;
  for (int s = 0; s < a.nsteps; s++) {
    cp_async_wait<kStage - 1>();  // step s's group is complete
    __syncwarp();
    if (!step(s)) {
      ok = false;
      break;
    }
    __syncwarp();  // every lane has read the slot before it is refilled
    issue(s + kStage);
  }
  cp_async_wait<0>();
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

// Dynamic shared memory of a launch: the rings, their minima and mbarriers, then the staging slots of its chains.
template <int LPT>
size_t chain_smem_bytes(int nw, int n, bool read_agg) {
  const size_t rings = (size_t)(kMaxChainWarps + 1) * kRingS * Dp_of(LPT) * 2 + (size_t)(kMaxChainWarps + 1) * kRingS * 2 + 16 +
                       (size_t)2 * (kMaxChainWarps + 1) * kRingS * 8;
  const size_t slot = ((size_t)n * (read_agg ? 3 : 1) + 8 + 15) & ~(size_t)15;
  return rings + (size_t)2 * nw * kStage * slot;
}

template <int LPT, bool FULL, bool PASS2, int GROUP>
void launch_chains_t(const SplitArgs& a, cudaStream_t s) {
  const int nw = chain_warps(a.nchains);
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
