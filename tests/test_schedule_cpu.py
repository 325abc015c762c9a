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
