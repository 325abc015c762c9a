// Device helpers of the uniform-layer aggregation kernels (sgm_uniform.cu: the fused four-path wavefront; sgm_split.cu:
// the path groups {0, 1} and {2, 3}): the kernel arguments, the packed-u16 plane vectors of a lane, one SGM path step
// (DenseStereoSgm.cs:276-313), and the loads and stores of raw costs, aggregates and revisit column states.
#pragma once
#include <cstdint>

#include "common.cuh"
#include "revisit_schedule.h"

namespace lux {

constexpr uint32_t kInit2 = 0x07d007d0u;  // 2000 | 2000: a never-written line-buffer word, twice

LUX_DEV uint32_t vmin2(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("min.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
LUX_DEV uint32_t pair_of(uint32_t lo_src_hi, uint32_t hi_src_lo) { return __byte_perm(lo_src_hi, hi_src_lo, 0x5432); }
LUX_DEV uint32_t dup16(uint32_t v) { return __byte_perm(v, 0, 0x1010); }

struct UniArgs {
  int W, H, n, T, dir, nCB;
  const uint8_t* raw;
  uint16_t* agg;
  float* depth;
  const float* planes;
  const uchar4* guidance;
  int p1;
  float p2base;
  float gw[4];
  uint16_t* bnd;      // [kBandBufs][W][3][Dp]
  uint16_t* bnd_min;  // [kBandBufs][W][3]
  int* progress;      // [nCB]
  int* ticket;
  uint16_t* edge;     // [W][3][Dp] pass +1's final half-0 row, unmirrored x (paths 1, 2, 3)
  uint16_t* edge_min; // [W][3]
  int y_b;            // its row, -1 = none
  int edge_write, edge_read;
  uint16_t* cs;       // [H][5][Dp] column states (rows of the pass)
  uint16_t* cs_min;   // [H][5]
  const int* flags;
  const int* batch_first;
  const int* batch_count;
  const int* src0;
  const int* src1;
  const int* src2;
  const int* extra;
  const uint2* p2t;   // [H][W] P2 of paths 0..3 per pixel of the pass
  int end_first, end_count;
  int keep_agg, wta;
  int* err;
  unsigned long long timeout_ns;
  int stall_block;    // failure-path tests: this block's cross-block wait reads `never` (-1: none)
  const int* never;
};

template <int LPT>
struct V {
  uint32_t r[LPT / 2];
};

template <int LPT>
LUX_DEV void vload(V<LPT>& v, const uint16_t* p, int lane) {
  const uint32_t* q = reinterpret_cast<const uint32_t*>(p + lane * LPT);
  if constexpr (LPT == 8) {
    uint4 t = __ldcg(reinterpret_cast<const uint4*>(q));
    v.r[0] = t.x; v.r[1] = t.y; v.r[2] = t.z; v.r[3] = t.w;
  } else if constexpr (LPT == 4) {
    uint2 t = __ldcg(reinterpret_cast<const uint2*>(q));
    v.r[0] = t.x; v.r[1] = t.y;
  } else if constexpr (LPT % 8 == 0) {  // LPT > 8: one 16-byte load per octet of planes
#pragma unroll
    for (int o = 0; o < LPT / 8; o++) {
      uint4 t = __ldcg(reinterpret_cast<const uint4*>(q) + o);
      v.r[4 * o] = t.x; v.r[4 * o + 1] = t.y; v.r[4 * o + 2] = t.z; v.r[4 * o + 3] = t.w;
    }
  } else {
    v.r[0] = __ldcg(q);
  }
}
template <int LPT>
LUX_DEV void vstore(const V<LPT>& v, uint16_t* p, int lane) {
  uint32_t* q = reinterpret_cast<uint32_t*>(p + lane * LPT);
  if constexpr (LPT == 8) __stcg(reinterpret_cast<uint4*>(q), make_uint4(v.r[0], v.r[1], v.r[2], v.r[3]));
  else if constexpr (LPT == 4) __stcg(reinterpret_cast<uint2*>(q), make_uint2(v.r[0], v.r[1]));
  else if constexpr (LPT % 8 == 0) {
#pragma unroll
    for (int o = 0; o < LPT / 8; o++)
      __stcg(reinterpret_cast<uint4*>(q) + o, make_uint4(v.r[4 * o], v.r[4 * o + 1], v.r[4 * o + 2], v.r[4 * o + 3]));
  } else __stcg(q, v.r[0]);
}
template <int LPT>
LUX_DEV void vload_s(V<LPT>& v, const uint16_t* p, int lane) {  // shared memory
  const uint32_t* q = reinterpret_cast<const uint32_t*>(p + lane * LPT);
#pragma unroll
  for (int i = 0; i < LPT / 2; i++) v.r[i] = q[i];
}
template <int LPT>
LUX_DEV void vstore_s(const V<LPT>& v, uint16_t* p, int lane) {
  uint32_t* q = reinterpret_cast<uint32_t*>(p + lane * LPT);
#pragma unroll
  for (int i = 0; i < LPT / 2; i++) q[i] = v.r[i];
}
template <int LPT>
LUX_DEV void vinit(V<LPT>& v) {
#pragma unroll
  for (int i = 0; i < LPT / 2; i++) v.r[i] = kInit2;
}

// A lane's planes in use, counted in octets (the plane count is a multiple of 8): the `active` argument of the helpers
// below. A lane of LPT <= 8 planes holds at most one octet, so it is 0 or 1 (any true value); past 256 planes (LPT 16 or
// 24) the last lane below the plane count may hold padding octets after its planes. Word i of a lane (planes 2i, 2i+1)
// is in use when i / 4 < active.
template <int LPT>
LUX_DEV int lane_octets(int n, int lane) {
  if constexpr (LPT <= 8) return lane * LPT < n ? 1 : 0;
  else return max(0, min(LPT / 8, (n - lane * LPT) / 8));
}

// One path step (DenseStereoSgm.cs:276-313) for a lane's planes. nb: the neighbour's L (2000 past the plane range),
// mp: its minimum, p2p: min(P2 + mp, 65535). Returns the new L; adds lc to acc; folds lc into rmin.
template <int LPT>
LUX_DEV void path_step(const V<LPT>& nb, uint32_t mp, uint32_t p2p, uint32_t p1x2, const V<LPT>& raw2, int active, int lane,
                       V<LPT>& out, V<LPT>& acc, uint32_t& rmin) {
  constexpr int NR = LPT / 2;
  uint32_t prev = __shfl_up_sync(0xffffffffu, nb.r[NR - 1], 1);
  uint32_t next = __shfl_down_sync(0xffffffffu, nb.r[0], 1);
  if (lane == 0) prev = kInit2;    // plane -1: the word before the block holds 2000
  if (lane == 31) next = kInit2;   // plane n (or a padding lane): 2000
  const uint32_t mp2 = dup16(mp), p2x2 = dup16(p2p);
  uint32_t lm[NR + 1];
  lm[0] = pair_of(prev, nb.r[0]);
#pragma unroll
  for (int i = 1; i < NR; i++) lm[i] = pair_of(nb.r[i - 1], nb.r[i]);
  lm[NR] = pair_of(nb.r[NR - 1], next);
#pragma unroll
  for (int i = 0; i < NR; i++) {
    uint32_t t = vmin2(lm[i], lm[i + 1]) + p1x2;       // min(L[d-1], L[d+1]) + P1
    t = vmin2(vmin2(t, nb.r[i]), p2x2);                 // with L[d] and P2 + minPrev
    uint32_t lc = t + raw2.r[i] - mp2;                   // raw + m - minPrev, each half in [0, 2000)
    lc = (i >> 2) < active ? lc : kInit2;                // padding planes keep 2000
    out.r[i] = lc;
    rmin = vmin2(rmin, lc);
    acc.r[i] += lc;
  }
}

template <int LPT>
LUX_DEV uint32_t warp_min(uint32_t rmin) {  // min over both halves and all lanes
  uint32_t m = min(rmin & 0xffffu, rmin >> 16);
  return __reduce_min_sync(0xffffffffu, m);
}

// The four paths of one pixel, written path-parallel so the independent chains interleave: all neighbour shuffles
// first, then the min/add chains, then the four warp minima. nb[p]/mp[p]: neighbour L and minimum of path p; p2[p]: P2.
template <int LPT, bool FULL>
LUX_DEV void four_paths(const V<LPT> (&nb)[4], const uint32_t (&mp)[4], const uint32_t (&p2)[4], uint32_t p1x2, const V<LPT>& raw2,
                        int active, int lane, V<LPT> (&out)[4], V<LPT>& acc, uint32_t (&mins)[4]) {
  constexpr int NR = LPT / 2;
  uint32_t prev[4], next[4];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    prev[p] = __shfl_up_sync(0xffffffffu, nb[p].r[NR - 1], 1);
    next[p] = __shfl_down_sync(0xffffffffu, nb[p].r[0], 1);
  }
  uint32_t rmin[4];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    if (lane == 0) prev[p] = kInit2;   // plane -1: the word before the block holds 2000
    if (lane == 31) next[p] = kInit2;  // plane n (or a padding lane): 2000
    rmin[p] = 0xffffffffu;
  }
#pragma unroll
  for (int i = 0; i < NR; i++) {
#pragma unroll
    for (int p = 0; p < 4; p++) {
      const uint32_t lm = pair_of(i == 0 ? prev[p] : nb[p].r[i - 1], nb[p].r[i]);       // L[d-1]
      const uint32_t lp = pair_of(nb[p].r[i], i == NR - 1 ? next[p] : nb[p].r[i + 1]);  // L[d+1]
      uint32_t t = vmin2(lm, lp) + p1x2;
      t = vmin2(vmin2(t, nb[p].r[i]), dup16(p2[p] + mp[p]));  // P2 <= 1744 and minPrev <= 2000: no u16 overflow
      uint32_t lc = t + raw2.r[i] - dup16(mp[p]);  // raw + m - minPrev, each half in [0, 2000)
      if (!FULL) lc = (i >> 2) < active ? lc : kInit2;  // padding planes keep 2000
      out[p].r[i] = lc;
      rmin[p] = vmin2(rmin[p], lc);
      acc.r[i] += lc;
    }
  }
#pragma unroll
  for (int p = 0; p < 4; p++) mins[p] = warp_min<LPT>(rmin[p]);
}

LUX_DEV float4 pix_of(const UniArgs& a, int xm, int ym) {  // guidance at a pixel given in pass coordinates
  const int x = a.dir > 0 ? xm : a.W - 1 - xm, y = a.dir > 0 ? ym : a.H - 1 - ym;
  const uchar4 g = __ldg(a.guidance + (size_t)y * a.W + x);
  return make_float4(g.x, g.y, g.z, g.w);
}
LUX_DEV float4 pix_edge(const UniArgs& a, int xu) {  // guidance of pass +1's row y_b at unmirrored x
  const uchar4 g = __ldg(a.guidance + (size_t)a.y_b * a.W + xu);
  return make_float4(g.x, g.y, g.z, g.w);
}
LUX_DEV int p2_of(const UniArgs& a, float4 g, float4 n) {
  const float gg[4] = {g.x, g.y, g.z, g.w}, nn[4] = {n.x, n.y, n.z, n.w};
  return sgm_p2(gg, nn, a.gw, a.p2base);
}

// A neighbour state: L vector, minimum and guidance.
template <int LPT>
struct Src {
  V<LPT> L;
  uint32_t mn;
  float4 pix;
};

template <int LPT>
LUX_DEV float4 pick_pix(const Src<LPT> (&s)[4], int lane) {  // lanes 0..3 take their path's neighbour guidance
  return lane == 0 ? s[0].pix : lane == 1 ? s[1].pix : lane == 2 ? s[2].pix : s[3].pix;
}

template <int LPT>
LUX_DEV void src_init(Src<LPT>& s) {
  vinit(s.L);
  s.mn = 2000;
  s.pix = make_float4(0.f, 0.f, 0.f, 0.f);
}
__host__ __device__ constexpr int Dp_of(int LPT) { return 32 * LPT; }

// The edge state (pass +1's final line buffer at row y_b) of path p (1..3) at unmirrored x.
template <int LPT>
LUX_DEV void src_edge(const UniArgs& a, Src<LPT>& s, int xu, int p, int lane) {
  if (a.y_b < 0 || xu < 0 || xu >= a.W) { src_init(s); return; }
  constexpr int Dp = Dp_of(LPT);
  vload<LPT>(s.L, a.edge + ((size_t)xu * 3 + (p - 1)) * Dp, lane);
  s.mn = __ldcg(a.edge_min + (size_t)xu * 3 + (p - 1));
  s.pix = pix_edge(a, xu);
}
// A column state of the revisit machinery.
template <int LPT>
LUX_DEV void src_cs(const UniArgs& a, Src<LPT>& s, int row, int slot, int xm, int lane) {
  constexpr int Dp = Dp_of(LPT);
  vload<LPT>(s.L, a.cs + ((size_t)row * 5 + slot) * Dp, lane);
  s.mn = __ldcg(a.cs_min + (size_t)row * 5 + slot);
  s.pix = pix_of(a, xm, row);
}
template <int LPT>
LUX_DEV void cs_put(const UniArgs& a, const V<LPT>& L, uint32_t mn, int row, int slot, int lane) {
  constexpr int Dp = Dp_of(LPT);
  vstore<LPT>(L, a.cs + ((size_t)row * 5 + slot) * Dp, lane);
  if (lane == 0) __stcg(a.cs_min + (size_t)row * 5 + slot, (uint16_t)mn);
}

template <int LPT>
LUX_DEV void load_raw(const UniArgs& a, int xm, int ym, V<LPT>& raw2, int active, int lane) {
  const int x = a.dir > 0 ? xm : a.W - 1 - xm, y = a.dir > 0 ? ym : a.H - 1 - ym;
  const uint8_t* p = a.raw + ((size_t)y * a.W + x) * a.n + lane * LPT;
  if (!active) {
#pragma unroll
    for (int i = 0; i < LPT / 2; i++) raw2.r[i] = 0;
    return;
  }
  if constexpr (LPT == 8) {
    uint2 b = __ldcs(reinterpret_cast<const uint2*>(p));
    raw2.r[0] = __byte_perm(b.x, 0, 0x4140); raw2.r[1] = __byte_perm(b.x, 0, 0x4342);
    raw2.r[2] = __byte_perm(b.y, 0, 0x4140); raw2.r[3] = __byte_perm(b.y, 0, 0x4342);
  } else if constexpr (LPT == 4) {
    uint32_t b = __ldcs(reinterpret_cast<const unsigned int*>(p));
    raw2.r[0] = __byte_perm(b, 0, 0x4140); raw2.r[1] = __byte_perm(b, 0, 0x4342);
  } else if constexpr (LPT % 8 == 0) {  // LPT > 8: the octets in use, 8 bytes each
#pragma unroll
    for (int o = 0; o < LPT / 8; o++) {
      uint2 b = o < active ? __ldcs(reinterpret_cast<const uint2*>(p) + o) : make_uint2(0u, 0u);
      raw2.r[4 * o] = __byte_perm(b.x, 0, 0x4140); raw2.r[4 * o + 1] = __byte_perm(b.x, 0, 0x4342);
      raw2.r[4 * o + 2] = __byte_perm(b.y, 0, 0x4140); raw2.r[4 * o + 3] = __byte_perm(b.y, 0, 0x4342);
    }
  } else {
    uint32_t b = __ldcs(reinterpret_cast<const unsigned short*>(p));
    raw2.r[0] = __byte_perm(b, 0, 0x4140);
  }
}

template <int LPT>
LUX_DEV uint16_t* agg_ptr(const UniArgs& a, int xm, int ym, int lane) {
  const int x = a.dir > 0 ? xm : a.W - 1 - xm, y = a.dir > 0 ? ym : a.H - 1 - ym;
  return a.agg + ((size_t)y * a.W + x) * a.n + lane * LPT;
}
template <int LPT>
LUX_DEV void agg_load(const uint16_t* p, V<LPT>& v, int active) {
  if (!active) {
#pragma unroll
    for (int i = 0; i < LPT / 2; i++) v.r[i] = 0;
    return;
  }
  if constexpr (LPT == 8) {
    uint4 t = __ldcs(reinterpret_cast<const uint4*>(p));
    v.r[0] = t.x; v.r[1] = t.y; v.r[2] = t.z; v.r[3] = t.w;
  } else if constexpr (LPT == 4) {
    uint2 t = __ldcs(reinterpret_cast<const uint2*>(p));
    v.r[0] = t.x; v.r[1] = t.y;
  } else if constexpr (LPT % 8 == 0) {  // LPT > 8: the octets in use (a padding octet would read the next pixel's planes)
#pragma unroll
    for (int o = 0; o < LPT / 8; o++) {
      uint4 t = o < active ? __ldcs(reinterpret_cast<const uint4*>(p) + o) : make_uint4(0u, 0u, 0u, 0u);
      v.r[4 * o] = t.x; v.r[4 * o + 1] = t.y; v.r[4 * o + 2] = t.z; v.r[4 * o + 3] = t.w;
    }
  } else {
    v.r[0] = __ldcs(reinterpret_cast<const unsigned int*>(p));
  }
}
template <int LPT>
LUX_DEV void agg_store(uint16_t* p, const V<LPT>& v, int active) {
  if (!active) return;
  if constexpr (LPT == 8) __stcs(reinterpret_cast<uint4*>(p), make_uint4(v.r[0], v.r[1], v.r[2], v.r[3]));
  else if constexpr (LPT == 4) __stcs(reinterpret_cast<uint2*>(p), make_uint2(v.r[0], v.r[1]));
  else if constexpr (LPT % 8 == 0) {  // LPT > 8: the octets in use only (the next pixel's planes follow)
#pragma unroll
    for (int o = 0; o < LPT / 8; o++)
      if (o < active) __stcs(reinterpret_cast<uint4*>(p) + o, make_uint4(v.r[4 * o], v.r[4 * o + 1], v.r[4 * o + 2], v.r[4 * o + 3]));
  } else __stcs(reinterpret_cast<unsigned int*>(p), v.r[0]);
}

// First minimum of the lane's planes, then over the warp (DenseStereoSgm.cs:228-230): key = value·4096 + plane.
template <int LPT>
LUX_DEV int wta_arg(const V<LPT>& agg, int active, int lane) {
  uint32_t best = 0xffffu, arg = 0xfffu;
  if (active) {
#pragma unroll
    for (int i = 0; i < LPT / 2; i++) {
      if ((i >> 2) >= active) break;  // padding planes of the lane
      uint32_t lo = agg.r[i] & 0xffffu, hi = agg.r[i] >> 16;
      if (lo < best) { best = lo; arg = lane * LPT + 2 * i; }
      if (hi < best) { best = hi; arg = lane * LPT + 2 * i + 1; }
    }
  }
  uint32_t key = __reduce_min_sync(0xffffffffu, (best << 12) | arg);
  return key >= (0xffffu << 12) ? 0 : (int)(key & 0xfffu);
}

// Raw bytes of a lane's planes as loaded (LPT, 4 or 2 bytes), unpacked to u16 pairs when used.
template <int LPT>
struct RawB {
  uint32_t r[LPT >= 8 ? LPT / 4 : 1];
};
template <int LPT>
LUX_DEV void raw_unpack(const RawB<LPT>& b, V<LPT>& raw2) {
  raw2.r[0] = __byte_perm(b.r[0], 0, 0x4140);
  if constexpr (LPT >= 4) raw2.r[1] = __byte_perm(b.r[0], 0, 0x4342);
  if constexpr (LPT >= 8) {
#pragma unroll
    for (int w = 1; w < LPT / 4; w++) {
      raw2.r[2 * w] = __byte_perm(b.r[w], 0, 0x4140);
      raw2.r[2 * w + 1] = __byte_perm(b.r[w], 0, 0x4342);
    }
  }
}

// A revisit R(c, y) (DenseStereoSgm.cs:234-317 replayed at the last column), run by one warp.
template <int LPT>
LUX_DEV void run_revisit(const UniArgs& a, int y, int lane, int active) {
  const int c = a.W - 1;
  Src<LPT> s[4];
  const int e[3] = {a.src0[y], a.src1[y], a.src2[y]};
  const int xsrc[3] = {c - 1, c - 1, c};
#pragma unroll
  for (int p = 0; p < 3; p++) {
    const int kind = src_kind(e[p]), row = src_row(e[p]);
    if (kind == kSrcInit) src_init(s[p]);
    else if (kind == kSrcEdge) src_edge<LPT>(a, s[p], a.dir > 0 ? xsrc[p] : a.W - 1 - xsrc[p], p, lane);
    else src_cs<LPT>(a, s[p], row, kind - kSrcCs, xsrc[p], lane);
  }
  src_init(s[3]);
  const float4 g = pix_of(a, c, y);
  int p2 = 0;
  if (lane < 4) p2 = p2_of(a, g, pick_pix<LPT>(s, lane));
  V<LPT> raw2, acc, out[4];
  load_raw<LPT>(a, c, y, raw2, active, lane);
#pragma unroll
  for (int i = 0; i < LPT / 2; i++) acc.r[i] = 0;
  const uint32_t p1x2 = dup16((uint32_t)a.p1);
  uint32_t mins[4];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    const int P2 = __shfl_sync(0xffffffffu, p2, p);
    const uint32_t p2p = (uint32_t)min(P2 + (int)s[p].mn, 65535);
    uint32_t rmin = 0xffffffffu;
    path_step<LPT>(s[p].L, s[p].mn, p2p, p1x2, raw2, active, lane, out[p], acc, rmin);
    mins[p] = warp_min<LPT>(rmin);
  }
  uint16_t* ap = agg_ptr<LPT>(a, c, y, lane);  // the revisit adds its four paths once more (:311)
  V<LPT> old;
  agg_load<LPT>(ap, old, active);
#pragma unroll
  for (int i = 0; i < LPT / 2; i++) old.r[i] += acc.r[i];
  agg_store<LPT>(ap, old, active);
  cs_put<LPT>(a, out[1], mins[1], y, 3, lane);
  cs_put<LPT>(a, out[2], mins[2], y, 4, lane);
  if (a.edge_write && (a.extra[y] & 1)) {  // R(y_b) is what pass -1 will read at the last column
    constexpr int Dp = Dp_of(LPT);
    vstore<LPT>(out[1], a.edge + ((size_t)c * 3 + 0) * Dp, lane);
    vstore<LPT>(out[2], a.edge + ((size_t)c * 3 + 1) * Dp, lane);
    if (lane == 0) {
      __stcg(a.edge_min + (size_t)c * 3 + 0, (uint16_t)mins[1]);
      __stcg(a.edge_min + (size_t)c * 3 + 1, (uint16_t)mins[2]);
    }
  }
  __syncwarp();
}

}  // namespace lux
