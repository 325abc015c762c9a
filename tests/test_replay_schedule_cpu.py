"""The exact replay's schedule (lux_b200/csrc/sgm_emulate.cu), checked on the CPU as a model of its waits.

The reference runs DenseLayer.Pixel() (DenseStereoSgm.cs:234-317) band by band, tile by tile, row by row, column by
column (DenseStereoSgm.cs:206-224), and its result depends on that order through the flat line buffer. The GPU replay
runs pixels concurrently: a band of T rows is split into parts (blocks) of min(8, T/2) rows, a warp per row, and each row goes
through its tiles on its own; row r runs offset u of tile i once row r-1 has finished it; a part's first row follows
the last row of the part above (same tile and offset within a band, offset u of tile i+1 across bands); waits at a
tile's start cover the revisits of the last column (a band's first row waits for the band above's revisits, all at
offset 0 of its last tile, before a tile that reaches column W-3). This test builds the happens-before graph of those waits and
checks that every two Pixel() calls that touch a common line-buffer region, one of them writing, are ordered as the
reference orders them, and that the graph has no cycle (no wait can deadlock).

A call's footprint, in the sheared column xp of its pass (memory order runs with xp in pass +1, against it in pass -1):
it writes its own slot (blocks and Min/Pix/Range entries) and spills past block 3 into the pad and first block-0
elements of the next slot in memory; it reads the other half's slots xp-1..xp+1 (each block window +-1 element, which
stays inside the blocks), the pad after its path-3 window, its own half's slot xp-1 (path 0, from that slot's pad) and
the Min/Pix/Range entries of those slots and its own.
"""
from collections import deque

import pytest


def _footprint(h, xp, dirn):
    hb = 1 - h
    nxt = (lambda c: c + 1) if dirn > 0 else (lambda c: c - 1)
    writes = {(h, "body", xp), (h, "meta", xp), (h, "pad", nxt(xp)), (h, "b0", nxt(xp))}
    reads = {(hb, "body", xp - 1), (hb, "body", xp), (hb, "body", xp + 1), (hb, "pad", nxt(xp + 1)),
             (h, "body", xp - 1), (h, "pad", xp - 1),
             (hb, "meta", xp - 1), (hb, "meta", xp), (hb, "meta", xp + 1), (h, "meta", xp - 1), (h, "meta", xp)}
    return writes, reads


def _pixel_xp(W, T, i, r, u):
    """The column of tile i's row r at offset u, or None (the kernel's emu_tile_pixel for rows inside the image)."""
    xs = min(max(i * T - r, 0), W - 1)
    xe = min(max(i * T + T - r, -1), W)
    if xs == xe:
        return None
    if i * T - r >= W:  # the clamped row start revisits the last column
        return W - 1 if u == 0 else None
    xp = i * T - r + u
    return xp if xs <= xp < xe else None


def _count_unordered(ids, preds, pixels):
    """Conflicting pairs of calls the happens-before graph leaves unordered against the reference's order, or -1 when
    the graph has a cycle."""
    n_nodes = len(ids)
    succ = [[] for _ in range(n_nodes)]
    indeg = [0] * n_nodes
    for b, ps in preds.items():
        for a in ps:
            succ[a].append(b)
            indeg[b] += 1
    queue, topo = deque(k for k in range(n_nodes) if indeg[k] == 0), []
    while queue:
        a = queue.popleft()
        topo.append(a)
        for b in succ[a]:
            indeg[b] -= 1
            if indeg[b] == 0:
                queue.append(b)
    if len(topo) != n_nodes:
        return -1
    before = [0] * n_nodes  # bitset of the nodes that happen before each node
    for b in topo:
        m = 0
        for a in preds.get(b, ()):
            m |= before[a] | (1 << a)
        before[b] = m
    pixels.sort(key=lambda p: p[0])
    touches = {}
    for idx, (_, _, (w, rd)) in enumerate(pixels):
        for g in w:
            touches.setdefault(g, []).append((idx, True))
        for g in rd:
            touches.setdefault(g, []).append((idx, False))
    bad = set()
    for lst in touches.values():
        for x in range(len(lst)):
            for y in range(x + 1, len(lst)):
                (ia, wa), (ib, wb) = lst[x], lst[y]
                if ia == ib or not (wa or wb):
                    continue
                a, b = min(ia, ib), max(ia, ib)
                if not (before[pixels[b][1]] >> pixels[a][1]) & 1:
                    bad.add((a, b))
    return len(bad)


def launcher_part_rows(T):
    """Rows per part (block) of a band, as the launcher splits it: min(8, T/2) rows for T >= 4, the whole band below."""
    return min(8, T // 2) if T >= 4 else T


def unordered_pairs(W, H, T, parts, dirn, lower_part_rule=False, own_part_rule=True, part_rows=None, band_reach=3):
    """Conflicting pairs the waits leave unordered (or -1 for a cycle). The band is split into parts of part_rows rows
    (the last part holds the rest: 8 + 8 + 8 + 8 + 2 at T = 34), or into `parts` equal parts when part_rows is None. A
    band's first row waits for the band above's revisits (offset 0 of its last tile) before a tile that reaches column
    W - band_reach (W - 3 in the kernel). Planted mistakes: lower_part_rule makes a lower part wait for the part above to
    finish its revisiting tile i+1 (instead of the part above waiting for it); own_part_rule=False drops the wait of a
    revisiting row for its own part's last row; band_reach=2 waits one column too late."""
    ghN, gwN = (H + T - 1) // T, (W + 2 * T - 1) // T
    R = part_rows if part_rows is not None else (T + parts - 1) // parts
    parts = (T + R - 1) // R
    ids, preds, pixels = {}, {}, []

    def node(key):
        if key not in ids:
            ids[key] = len(ids)
        return ids[key]

    def edge(a, b):
        preds.setdefault(b, set()).add(a)

    def pub_row(j, part):
        return min(part * R + R, T, H - j * T) - 1

    for j in range(ghN):
        for part in range(parts):
            r0, r1 = part * R, min(part * R + R, T)
            if j * T + r0 >= H:
                continue  # a part below the image returns at once
            rows = [r for r in range(r0, r1) if j * T + r < H]
            rp = pub_row(j, part)
            for r in rows:
                for i in range(gwN):
                    for u in range(T):
                        n = node((j, part, r, i, u))
                        if u > 0:
                            edge(node((j, part, r, i, u - 1)), n)
                        elif i > 0:  # the row's own previous tile
                            edge(node((j, part, r, i - 1, T - 1)), n)
                        if r > r0:  # the row above in this part through offset u
                            edge(node((j, part, r - 1, i, u)), n)
                        if r == r0 and (j, part) != (0, 0):  # the part above's last row
                            if part > 0:
                                key = (j, part - 1, pub_row(j, part - 1), i, u)
                            else:
                                tgt = min((i + 1) * T + u + 1, gwN * T)
                                key = (j - 1, parts - 1, pub_row(j - 1, parts - 1), (tgt - 1) // T, (tgt - 1) % T)
                            edge(node(key), n)
                        if u == 0:  # waits at the tile's start
                            waits = []
                            if r == r0 and part == 0 and j > 0 and (i + 1) * T >= W - band_reach + 1:
                                edge(node((j - 1, parts - 1, pub_row(j - 1, parts - 1), gwN - 1, 0)), n)
                            if lower_part_rule:
                                if r == r0 and part > 0 and (i + 1) * T - (r0 - R) >= W:
                                    waits.append((j, part - 1, min(i + 2, gwN) - 1))
                            elif r == r0 and part + 1 < parts and i > 0 and i * T - r0 >= W and j * T + r1 < H:
                                last = min(parts - 1, (H - j * T - 1) // R)  # the band's last part with rows in the image
                                waits.append((j, last, i - 1))
                            if own_part_rule and i > 0 and i * T - r >= W and r != rp:
                                waits.append((j, part, i - 1))
                            for (pj, pp, ti) in waits:
                                edge(node((pj, pp, pub_row(pj, pp), ti, T - 1)), n)
                        xp = _pixel_xp(W, T, i, r, u)
                        if xp is not None:
                            ref = (j, i, r, u if i * T - r < W else 0)
                            pixels.append((ref, n, _footprint(1 if r % 2 == 0 else 0, xp, dirn)))
    return _count_unordered(ids, preds, pixels)


def unordered_pairs_barrier_form(W, H, T, dirn, lag=3):
    """The same check for the barrier form (odd tiles, tiles past 64 rows): one block per band, pixel (r, u) of a tile at
    step u + 2r with a block barrier after every step and tile, a band starting tile i once the band above finished tile
    i + lag - 1 (lag 3 in the kernel)."""
    ghN, gwN = (H + T - 1) // T, (W + 2 * T - 1) // T
    ids, preds, pixels = {}, {}, []

    def node(key):
        if key not in ids:
            ids[key] = len(ids)
        return ids[key]

    def edge(a, b):
        preds.setdefault(b, set()).add(a)

    steps = 3 * T - 2
    for j in range(ghN):
        for i in range(gwN):
            start = node((j, i, "start"))
            if i > 0:
                edge(node((j, i - 1, "step", steps - 1)), start)
            if j > 0:
                edge(node((j - 1, min(i + lag - 1, gwN - 1), "step", steps - 1)), start)
            prev = start
            for t in range(steps):
                done = node((j, i, "step", t))
                for r in range(max(0, (t - T + 2) // 2), min(T - 1, t // 2) + 1):
                    u = t - 2 * r
                    if j * T + r >= H:
                        continue
                    xp = _pixel_xp(W, T, i, r, u)
                    if xp is None:
                        continue
                    n = node((j, i, r, u))
                    edge(prev, n)
                    edge(n, done)
                    pixels.append(((j, i, r, u if i * T - r < W else 0), n, _footprint(1 if r % 2 == 0 else 0, xp, dirn)))
                edge(prev, done)
                prev = done
    return _count_unordered(ids, preds, pixels)


@pytest.mark.parametrize("W,H,T", [(65, 49, 4), (48, 40, 8), (97, 61, 16), (70, 45, 32), (66, 65, 64), (33, 17, 2),
                                   (40, 10, 4), (20, 11, 6), (75, 70, 34), (83, 90, 40), (61, 55, 50), (90, 130, 62)])
@pytest.mark.parametrize("dirn", [1, -1])
def test_replay_waits_keep_the_reference_order(W, H, T, dirn):
    """Even tiles whose band the launcher splits into parts of min(8, T/2) rows, including the tiles that are not
    multiples of 8, where the last part is shorter (T = 34: four parts of 8 and one of 2; T = 50: six of 8 and one of 2)."""
    assert unordered_pairs(W, H, T, 0, dirn, part_rows=launcher_part_rows(T)) == 0


def test_order_check_catches_a_wrong_revisit_rule():
    """A lower part that waits for the upper part's revisiting tile i+1 runs the reference's order backwards there, and
    a revisiting row that does not wait for the rows below it in its part overtakes their previous tile."""
    assert unordered_pairs(65, 49, 4, 2, 1, lower_part_rule=True) > 0
    assert unordered_pairs(30, 20, 4, 2, -1, lower_part_rule=True) > 0
    assert unordered_pairs(70, 45, 32, 2, 1, own_part_rule=False) > 0
    assert unordered_pairs(40, 10, 4, 2, -1, own_part_rule=False) > 0


@pytest.mark.parametrize("W,H,T,dirn", [(66, 65, 64, 1), (130, 98, 16, 1), (66, 40, 4, 1)])
def test_order_check_catches_a_late_band_wait(W, H, T, dirn):
    """A band whose first row waits for the band above's revisits only before a tile reaching column W-2 (one column
    late) writes the slots that those revisits still read."""
    assert unordered_pairs(W, H, T, 0, dirn, part_rows=launcher_part_rows(T), band_reach=2) > 0
    assert unordered_pairs(W, H, T, 0, dirn, part_rows=launcher_part_rows(T)) == 0


@pytest.mark.parametrize("W,H,T,dirn", [(66, 65, 64, 1), (130, 100, 64, -1), (70, 45, 32, 1), (83, 90, 40, -1)])
def test_shorter_parts_keep_the_reference_order(W, H, T, dirn):
    """Parts of 4 rows (up to 16 a band) and 16 rows: the waits do not depend on the part size."""
    assert unordered_pairs(W, H, T, 0, dirn, part_rows=4) == 0
    assert unordered_pairs(W, H, T, 0, dirn, part_rows=16) == 0


def test_four_parts_wait_for_the_last_part():
    """With more than two parts, a revisiting part must wait for the band's last part, not only the next one down."""
    assert unordered_pairs(66, 65, 64, 4, 1) == 0
    assert unordered_pairs(66, 100, 64, 4, -1) == 0


def test_odd_tiles_need_the_barrier_form():
    """With an odd T a band's last row and the next band's first row share a line-buffer half, and the row form's
    hand-over leaves a conflicting pair unordered there: the launcher gives odd tiles the barrier form."""
    assert unordered_pairs(20, 11, 3, 1, 1) > 0


@pytest.mark.parametrize("W,H,T", [(20, 11, 3), (41, 30, 5), (23, 16, 3)])
@pytest.mark.parametrize("dirn", [1, -1])
def test_barrier_form_keeps_the_reference_order(W, H, T, dirn):
    assert unordered_pairs_barrier_form(W, H, T, dirn) == 0


def test_barrier_form_needs_its_band_lag():
    """A one-tile band lag lets a band run beside the band above's next tile, which an odd tile's shared half forbids."""
    assert unordered_pairs_barrier_form(20, 11, 3, 1, lag=1) > 0
