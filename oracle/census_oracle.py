"""CPU restatement (test infrastructure) of the opt-in census stereo mode: census transform, Hamming matching cost,
8-path semi-global aggregation with constant penalties, winner-take-all with parabolic subpixel refinement and a
left/right consistency check, and the fusion of per-pair disparities into one depth map.

The reference (Lux.Engine) has no such stage: its dense stage is a multi-view plane sweep (DenseStereo.cs,
DenseStereoSgm.cs). This mode follows the published semi-global matching method (Hirschmueller, "Stereo Processing by
Semiglobal Matching and Mutual Information", PAMI 2008) with the census transform of Zabih and Woodfill (ECCV 1994), with
the conventions fixed below. Parity unpinned: the GPU kernels are checked against this restatement only.

Conventions
  census:   9x7 window (x +-4, y +-3), 62 bits in row-major order of the neighbours (the centre skipped), bit k set when
            the neighbour is darker than the centre; neighbours outside the image are read at the clamped position.
  cost:     C(x, y, d) = popcount(census_L(x, y) XOR census_R(x - d, y)) for x - d >= 0, else 62, d in [0, D).
  paths:    the eight directions (+-1, 0), (0, +-1), (+-1, +-1); along each,
            L(p, d) = C(p, d) + min(L(q, d), L(q, d-1) + P1, L(q, d+1) + P1, min_k L(q, k) + P2) - min_k L(q, k)
            with q = p - r the previous pixel of the path (L(p) = C(p) where q is outside the image); S = sum of the eight.
  WTA:      d* = the first d with the least S; subpixel d* + (S[d*-1] - S[d*+1]) / (2 (S[d*-1] - 2 S[d*] + S[d*+1])) when
            0 < d* < D - 1 and the denominator is positive (float32), else d*.
  L/R:      d*_R(x) = the first d with the least S(x + d, y, d) over x + d < W; a pixel keeps its disparity when
            |d*(x) - d*_R(x - d*(x))| <= lr_max_diff, else gets -1.
  fusion:   per pair depth z = fB / disparity where disparity > 0; the fused depth is the median of a pixel's valid depths
            (the mean of the two middle ones for an even count, in float32), 0 where none is valid.
"""
import numpy as np

WX, WY = 4, 3
INVALID_COST = 62


def census(img):
    """(h, w) uint8 -> (h, w) uint64."""
    im = np.asarray(img, np.int32)
    h, w = im.shape
    out = np.zeros((h, w), np.uint64)
    bit = 0
    ys, xs = np.arange(h), np.arange(w)
    for dy in range(-WY, WY + 1):
        for dx in range(-WX, WX + 1):
            if dx == 0 and dy == 0:
                continue
            nb = im[np.clip(ys + dy, 0, h - 1)][:, np.clip(xs + dx, 0, w - 1)]
            out |= (nb < im).astype(np.uint64) << np.uint64(bit)
            bit += 1
    return out


def _popcount64(v):
    v = v.astype(np.uint64)
    c = np.zeros(v.shape, np.uint8)
    for s in range(0, 64, 8):
        b = ((v >> np.uint64(s)) & np.uint64(0xFF)).astype(np.uint8)
        c += np.unpackbits(b[..., None], axis=-1).sum(-1).astype(np.uint8)
    return c


def hamming_cost(cl, cr, D):
    """(h, w, D) uint8 matching cost."""
    h, w = cl.shape
    C = np.full((h, w, D), INVALID_COST, np.uint8)
    for d in range(D):
        if d < w:
            C[:, d:, d] = _popcount64(cl[:, d:] ^ cr[:, :w - d])
    return C


def _step(Lq, Cp, P1, P2):
    """One path step for a batch: Lq, Cp (n, D) int32 -> (n, D)."""
    big = 1 << 20
    m = Lq.min(1, keepdims=True)
    lm = np.concatenate([np.full((Lq.shape[0], 1), big), Lq[:, :-1]], 1) + P1
    lp = np.concatenate([Lq[:, 1:], np.full((Lq.shape[0], 1), big)], 1) + P1
    t = np.minimum(np.minimum(Lq, lm), np.minimum(lp, m + P2))
    return Cp + t - m


def aggregate(C, P1, P2):
    """S (h, w, D) int32: the sum of the eight path costs."""
    h, w, D = C.shape
    C = C.astype(np.int32)
    S = np.zeros((h, w, D), np.int64)
    for dx, dy in ((1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (-1, -1), (1, -1), (-1, 1)):
        L = np.zeros((h, w, D), np.int64)
        if dy == 0:  # columns in path order, all rows at once
            order = range(w) if dx > 0 else range(w - 1, -1, -1)
            prev = None
            for x in order:
                L[:, x] = C[:, x] if prev is None else _step(L[:, prev], C[:, x], P1, P2)
                prev = x
        else:  # rows in path order, all columns at once; the previous pixel is one row back and dx columns left
            order = range(h) if dy > 0 else range(h - 1, -1, -1)
            prev = None
            for y in order:
                if prev is None:
                    L[y] = C[y]
                else:
                    xs = np.arange(w)
                    q = xs - dx
                    inside = (q >= 0) & (q < w)
                    L[y] = C[y]
                    if inside.any():
                        L[y, inside] = _step(L[prev, q[inside]], C[y, inside], P1, P2)
                prev = y
        S += L
    return S.astype(np.int32)


def wta(S, lr_max_diff=1, subpixel=True, lr_check=True):
    """(h, w) float32 disparities (-1 where the left/right check fails)."""
    h, w, D = S.shape
    dl = S.argmin(2)
    out = dl.astype(np.float32)
    if subpixel:
        ys, xs = np.mgrid[0:h, 0:w]
        inner = (dl > 0) & (dl < D - 1)
        dm = np.where(inner, dl - 1, 0)
        dp = np.where(inner, dl + 1, 0)
        a = S[ys, xs, dm].astype(np.float32)
        b = S[ys, xs, dl].astype(np.float32)
        c = S[ys, xs, dp].astype(np.float32)
        den = np.float32(2.0) * ((a - np.float32(2.0) * b) + c)
        ok = inner & (den > 0)
        corr = np.where(ok, (a - c) / np.where(ok, den, np.float32(1.0)), np.float32(0.0)).astype(np.float32)
        out = (dl.astype(np.float32) + corr).astype(np.float32)
    if lr_check:
        dr = np.zeros((h, w), np.int64)
        for x in range(w):
            dmax = min(D, w - x)
            vals = np.stack([S[:, x + d, d] for d in range(dmax)], 1)
            dr[:, x] = vals.argmin(1)
        xr = np.arange(w)[None, :] - dl
        valid = xr >= 0
        drr = np.where(valid, dr[np.arange(h)[:, None], np.clip(xr, 0, w - 1)], 1 << 20)
        bad = ~valid | (np.abs(dl - drr) > lr_max_diff)
        out = np.where(bad, np.float32(-1.0), out).astype(np.float32)
    return out


def census_sgm(left, right, D, P1, P2, lr_max_diff=1, subpixel=True, lr_check=True):
    cl, cr = census(left), census(right)
    S = aggregate(hamming_cost(cl, cr, D), P1, P2)
    return wta(S, lr_max_diff, subpixel, lr_check)


def fuse(disps, fbs):
    """Median depth over the pairs' valid disparities (float32), 0 where none is valid."""
    disp = np.stack([np.asarray(d, np.float32) for d in disps], 0)
    fb = np.asarray(fbs, np.float32)[:, None, None]
    z = np.where(disp > 0, fb / np.where(disp > 0, disp, np.float32(1.0)), np.float32(np.nan)).astype(np.float32)
    zs = np.sort(z, 0)  # NaN last
    n = np.isfinite(zs).sum(0)
    out = np.zeros(disp.shape[1:], np.float32)
    for k in range(1, disp.shape[0] + 1):
        sel = n == k
        if not sel.any():
            continue
        if k % 2:
            out[sel] = zs[k // 2][sel]
        else:
            out[sel] = ((zs[k // 2 - 1][sel] + zs[k // 2][sel]) * np.float32(0.5)).astype(np.float32)
    return out
