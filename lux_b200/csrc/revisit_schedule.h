// The revisit schedule of a uniform layer: which reads of the reference's line buffers (DenseStereoSgm.cs:206-224)
// deviate from a plain raster recurrence, and what they read instead.
//
// Coordinates are those of the pass (mirrored for pass -1: x' = W-1-x, y' = H-1-y). With T even, a row's half of
// the line buffer is the parity of its row, so a plain recurrence gives every read its raster neighbour, except:
//   * the last column c = W-1 of rows r < K = T - ((W-1) mod T) of each T-row band is visited a second time ("R",
//     after the band's tile that holds the column), reading whatever the neighbour slots hold by then;
//   * path 2 of the normal visit N(c, y) reads R(c, y-1) instead of N(c, y-1) when y is the first row of the band's
//     last tile (r = K < rows) or when y starts a band after a band with K = T;
//   * pass -1 starts from the line buffer pass +1 left: its row -1 is pass +1's last odd row (y_b), whose last-column
//     slot may hold R(y_b).
// Path 0, 1 and 3 of every normal visit read their raster neighbours (a revisit's path 3 restarts from the margin
// exactly like the normal visit does, so its value equals the normal one).
#pragma once
#include <algorithm>
#include <cstdint>
#include <vector>

namespace lux {

// source kinds of a revisit's neighbour read
enum : int {
  kSrcInit = 0,  // a never-written slot: L = 2000, Min = 2000, Pix = 0
  kSrcEdge = 1,  // pass +1's final line buffer (pass -1 only)
  kSrcCs = 2,    // a per-row column state, slot (kind - kSrcCs): 0 N(c-1).p0, 1 N(c-1).p1, 2 N(c).p2, 3 R(c).p1, 4 R(c).p2
};
#ifdef __CUDACC__
#define LUX_HD __host__ __device__
#else
#define LUX_HD
#endif
LUX_HD inline int src_enc(int kind, int row) { return (kind << 24) | (row & 0xffffff); }
LUX_HD inline int src_kind(int e) { return e >> 24; }
LUX_HD inline int src_row(int e) { return e & 0xffffff; }

struct RevisitSchedule {
  // per row of the pass: flags bit 0: N(c).p2 reads R(c, y-1). batch_first / batch_count: the revisit rows this row
  // runs just before its own N(c) (count 0 = none).
  std::vector<int> flags, batch_first, batch_count;
  // the last band's revisits when it has no row after them: run by the last row after its own N(c)
  int end_first = 0, end_count = 0;
  // per row with a revisit: the sources of paths 0, 1, 2 (path 3 reads the margin), and bit 0 of extra = this revisit
  // is the last writer of the last column's half-0 slot at the end of pass +1.
  std::vector<int> src0, src1, src2, extra;
  int y_b = -1;  // pass +1's last odd row (pass -1's row -1), -1 if none
};

// second_pass: the sources that fall off band 0 read pass +1's final state (kSrcEdge) instead of kSrcInit.
inline void build_revisit_schedule(int W, int H, int T, bool second_pass, RevisitSchedule& s) {
  const int K = T - (W - 1) % T;
  const int nb = (H + T - 1) / T;
  s.flags.assign(H, 0);
  s.end_first = 0;
  s.end_count = 0;
  s.batch_first.assign(H, 0);
  s.batch_count.assign(H, 0);
  s.src0.assign(H, 0);
  s.src1.assign(H, 0);
  s.src2.assign(H, 0);
  s.extra.assign(H, 0);
  const int boundary = src_enc(second_pass ? kSrcEdge : kSrcInit, 0);
  auto rows_of = [&](int j) { return std::min(T, H - j * T); };
  for (int j = 0; j < nb; j++) {
    const int nr = rows_of(j), base = j * T;
    for (int r = 0; r < nr; r++)
      if ((r == K && K < nr) || (r == 0 && j > 0 && K == T)) s.flags[base + r] |= 1;
    const int nrev = std::min(K, nr);
    if (nrev <= 0) continue;
    if (K < nr || j + 1 < nb) {
      const int exec = K < nr ? base + K : (j + 1) * T;
      s.batch_first[exec] = base;
      s.batch_count[exec] = nrev;
    } else {
      s.end_first = base;
      s.end_count = nrev;
    }
    const int lim = std::min(std::min(K, T - 1), nr - 1);  // rows that visit column c-1 before the band's last tile
    for (int r = 0; r < nrev; r++) {
      const int y = base + r;
      if (W >= 2) {
        const int r0 = lim - ((lim - r) & 1);
        s.src0[y] = src_enc(kSrcCs + 0, base + r0);
        const int q = (r + 1) & 1;
        if (lim >= q) s.src1[y] = src_enc(kSrcCs + 1, base + (lim - ((lim - q) & 1)));
        else s.src1[y] = j > 0 ? src_enc(kSrcCs + 1, base - 1) : boundary;
      } else {
        s.src0[y] = src_enc(kSrcInit, 0);
        s.src1[y] = src_enc(kSrcInit, 0);
      }
      if (r >= 1) {
        s.src2[y] = src_enc(kSrcCs + 4, y - 1);
      } else {
        const int m = std::min(K, nr) - 1;  // the last row of the band visited in the column's own tile
        if (m >= 1) s.src2[y] = src_enc(kSrcCs + 2, base + (m - ((m + 1) & 1)));
        else if (j > 0) s.src2[y] = src_enc(K < T ? kSrcCs + 2 : kSrcCs + 4, base - 1);
        else s.src2[y] = boundary;
      }
    }
  }
  s.y_b = H >= 2 ? ((H - 1) % 2 == 1 ? H - 1 : H - 2) : -1;
  if (!second_pass && s.y_b >= 0) {
    const int jb = s.y_b / T, rb = s.y_b % T;
    if (rb < std::min(K, rows_of(jb))) s.extra[s.y_b] |= 1;
  }
}

}  // namespace lux
