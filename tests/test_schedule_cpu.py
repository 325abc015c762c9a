"""CPU proof obligations of the GPU traversal replay (lux_b200/csrc/sgm_emulate.cu).

The reference aggregates with a strictly sequential sweep (DenseStereoSgm.cs:206-224). The GPU replays every Pixel()
call of that sweep but runs many at once: bands of T rows are pipelined (band j starts tile i once band j-1 finished
tile i+2) and inside a tile pixel (r, u) runs at step u + 2r. This test replays the reference order from the oracle's
traversal trace and checks, for every pair of calls that touch a common line-buffer slot (and at least one writes it),
that the GPU schedule runs them in the reference's order and never in the same step.
"""
import numpy as np
import pytest


def _key(ev, W, H, T):
    d, x, y, r, rev = (int(v) for v in ev[:5])
    xp = x if d > 0 else W - 1 - x
    yp = y if d > 0 else H - 1 - y
    j = yp // T
    if rev:
        i, u = (xp + r) // T + 1, 0
    else:
        i = (xp + r) // T
        u = xp + r - i * T
    return (0 if d > 0 else 1, j, i, u + 2 * r)


def _ordered(a, b):
    """True when the GPU schedule runs call a strictly before call b."""
    if a[0] != b[0]:
        return a[0] < b[0]  # the passes are separate launches
    if a[1] == b[1]:
        return (a[2], a[3]) < (b[2], b[3])
    if a[1] < b[1]:
        return a[2] <= b[2] + 2 * (b[1] - a[1])
    return False


def _check(oracle, W, H, T):
    tr = oracle.traversal_trace(W, H, T)
    keys = [_key(e, W, H, T) for e in tr]
    last_w = {}
    readers = {}
    bad = []
    for n, e in enumerate(tr):
        d, x, r = int(e[0]), int(e[1]), int(e[3])
        s = x + 1
        cur = 1 if (r & 1) == 0 else 0
        oth = 1 - cur
        wr = {(cur, s), (cur, s + 1)}                   # own slot and the spill into the next slot
        rd = set()
        for half, ns in ((cur, s - d), (oth, s - d), (oth, s), (oth, s + d)):
            rd.add((half, ns))
            rd.add((half, ns + 1))                      # reads past a block reach the next slot's first words
        for k in rd - wr:
            w = last_w.get(k)
            if w is not None and not _ordered(keys[w], keys[n]):
                bad.append(("RAW", k, w, n))
            readers.setdefault(k, []).append(n)
        for k in wr:
            w = last_w.get(k)
            if w is not None and w != n and not _ordered(keys[w], keys[n]):
                bad.append(("WAW", k, w, n))
            for q in readers.get(k, []):
                if q != n and not _ordered(keys[q], keys[n]):
                    bad.append(("WAR", k, q, n))
            last_w[k] = n
            readers[k] = []
    return bad


@pytest.mark.parametrize("T", [2, 4, 8, 16])
def test_replay_schedule_keeps_reference_order(oracle, T):
    sizes = [(1, 1), (2, 3), (3, 2), (5, 7), (9, 9), (17, 9), (20, 13), (22, 10), (25, 16), (33, 21), (40, 30), (65, 49)]
    for W, H in sizes:
        bad = _check(oracle, W, H, T)
        assert not bad, (W, H, T, bad[:5])


def test_revisits_exist_where_the_reference_has_them(oracle):
    """The sheared tiles visit the last column twice in pass +1 (column 0 in pass -1) for tile rows r < T - ((W-1) mod T)."""
    for W, H, T in [(20, 13, 4), (17, 9, 4), (65, 49, 4), (40, 30, 8)]:
        tr = oracle.traversal_trace(W, H, T)
        rev = tr[tr[:, 4] == 1]
        k = T - (W - 1) % T
        exp = sum(min(k, min(T, H - j * T)) for j in range((H + T - 1) // T))
        assert (rev[:, 0] == 1).sum() == exp and (rev[:, 0] == -1).sum() == exp
        assert (rev[rev[:, 0] == 1][:, 1] == W - 1).all() and (rev[rev[:, 0] == -1][:, 1] == 0).all()


def _sched_checks(oracle, W, H, T):
    """The fast uniform kernel's revisit schedule (lux_sgm_revisit_schedule) against the reference traversal."""
    from lux_b200 import api
    tr = oracle.traversal_trace(W, H, T)
    n1 = int((tr[:, 0] == 1).sum())
    sched = [api.revisit_schedule(W, H, T, False), api.revisit_schedule(W, H, T, True)]
    y_b = sched[0][1]
    bad = []
    for pi, d in enumerate((1, -1)):
        s = sched[pi][0]
        end_first, end_count = sched[pi][2]
        lo, hi = (0, n1) if d > 0 else (n1, len(tr))
        cu = W - 1 if d > 0 else 0
        ym = (lambda y: y) if d > 0 else (lambda y: H - 1 - y)
        xm = (lambda x: x) if d > 0 else (lambda x: W - 1 - x)
        c = W - 1
        n_seen = set()
        for n in range(lo, hi):
            dd, x, y, r, rev = (int(v) for v in tr[n][:5])
            srcs = [int(v) for v in tr[n][5:9]]
            if x != cu:
                continue
            if rev:
                # executor: every N at the column that precedes this revisit is a row above the executor
                exp = []
                for p in range(3):
                    e = srcs[p]
                    if e < 0:
                        exp.append(0)
                    elif int(tr[e][0]) != d:
                        exp.append(1 << 24)
                    else:
                        ex, ey, erv = int(tr[e][1]), int(tr[e][2]), int(tr[e][4])
                        slot = {0: 0, 1: 1}[p] if p < 2 else (4 if erv else 2)
                        want_x = c - 1 if p < 2 else c
                        if xm(ex) != want_x or (p < 2 and erv):
                            bad.append(("src pixel", d, y, p, ex, ey))
                        exp.append(((2 + slot) << 24) | ym(ey))
                got = [int(s[ym(y)][3]), int(s[ym(y)][4]), int(s[ym(y)][5])]
                if got != exp:
                    bad.append(("sources", d, y, got, exp))
                if srcs[3] != -1:
                    bad.append(("p3", d, y))
                ex_rows = [(yy, False) for yy in range(H) if s[yy][2] > 0 and s[yy][1] <= ym(y) < s[yy][1] + s[yy][2]]
                if end_first <= ym(y) < end_first + end_count:
                    ex_rows.append((H - 1, True))
                if len(ex_rows) != 1:
                    bad.append(("executor count", d, y, ex_rows))
                else:
                    e_row, after = ex_rows[0]
                    before_rows = {q for q in n_seen}
                    want = set(range(e_row + 1)) if after else set(range(e_row))
                    if before_rows != want:
                        bad.append(("executor order", d, y, e_row, after, sorted(before_rows - want), sorted(want - before_rows)))
            else:
                n_seen.add(ym(y))
                e = srcs[2]
                special = bool(s[ym(y)][0] & 1)
                is_r = e >= 0 and int(tr[e][0]) == d and int(tr[e][4]) == 1
                if special != is_r:
                    bad.append(("N p2", d, y, special, is_r))
    # pass -1's first row reads pass +1's final half-0 slots: row y_b, and R(y_b) at the last column when flagged
    s0 = sched[0][0]
    for n in range(n1, len(tr)):
        dd, x, y, r, rev = (int(v) for v in tr[n][:5])
        if y != H - 1 or rev:
            continue
        for p in (1, 2, 3):
            e = int(tr[n][5 + p])
            if e < 0 or int(tr[e][0]) != 1:
                continue
            ex, ey, erv = int(tr[e][1]), int(tr[e][2]), int(tr[e][4])
            if ey != y_b:
                bad.append(("edge row", x, p, ey, y_b))
            if erv and not (ex == W - 1 and (s0[y_b][6] & 1)):
                bad.append(("edge revisit", x, p))
            if not erv and ex == W - 1 and (s0[y_b][6] & 1):
                bad.append(("edge normal", x, p))
    return bad


@pytest.mark.parametrize("T", [2, 4, 8, 16, 64])
def test_revisit_schedule_matches_reference_traversal(oracle, T):
    sizes = [(3, 2), (5, 7), (9, 9), (17, 9), (20, 13), (22, 10), (25, 16), (33, 21), (40, 30), (65, 49), (66, 3), (130, 70)]
    for W, H in sizes:
        bad = _sched_checks(oracle, W, H, T)
        assert not bad, (W, H, T, bad[:4])
